// canon_sparse.cuh -- one warp canonizes one graph of any size (n <= 65536).
//
// Same search as canon_warp64.cuh -- the reference's sequential DFS
// (src/sequential.cpp:216-670) step for step, bit-exact in canonical form,
// stored automorphisms and node count -- with data structures whose cost
// follows the work a step does rather than n:
//
//   * the ordered partition is elem[] / pos[] plus a two-level bitmap of cell
//     start positions; a vertex's cell is the last start at or before its
//     position, so splitting a cell only sets bits and swaps the moved
//     vertices, and backtracking (reconstruct_at_level) only clears bits;
//   * a refinement step touches only the neighbours of the splitter: counts
//     go to cnt[], touched vertices are grouped per cell by a counting sort,
//     and each split cell is rearranged by pairing its misplaced vertices
//     with the holes of the target region -- O(touched), the work nauty does;
//   * a leaf certificate is, per vertex, the sorted canonical positions of
//     its neighbours (O(m) words), compared row by row in canonical order
//     exactly like the upper-triangle compare (sequential.cpp:114-124);
//   * the target cell of a level is not stored: when the search is back at
//     that level the partition is the same, so its members are the cell at
//     the stored start position; orbit representatives live in a small
//     stack of per-level arrays that are only allocated when orbits are
//     first computed at a level.
//
// All state lives in a per-warp slot of device memory; the warp's pointers
// and scalars live in shared memory.  Each phase is one non-inlined function.
#pragma once
#include <cstdint>

#include "canon_warp64.cuh"
#include "gcl_device.cuh"

namespace gcl {

constexpr int kSpThreads = 128;
constexpr int kSpWarps = kSpThreads / 32;
constexpr uint32_t kNone = 0xffffffffu;

struct SpTc {
  uint32_t first, len, counter;
  int32_t last;   // last_num_aut_at_level
  int32_t rslot;  // slot of this level's representatives, -1 = all v are reps
  uint32_t pad;
};

// Byte layout of one slot for graphs with at most n vertices and m2 CSR
// entries, `pool` per-level representative arrays and `cap` ring slots.
struct SpLayout {
  uint64_t u32n[26];  // offsets of the n-sized u32 arrays
  uint64_t fcode, ccode, pool_owner;
  uint64_t stb, sts, act, acts, tcb, tcbs;
  uint64_t fcert, bcert, ccert;
  uint64_t tc, reps, auts, ulog, fixst;
  uint32_t ulog_cap, fixcap;
  uint64_t bytes;
  uint32_t nw, nsw;
  uint32_t stride;  // elements per representative array / ring entry
};

__host__ __device__ inline SpLayout sp_layout(uint32_t n, uint64_t m2, uint32_t pool,
                                              uint32_t cap, uint32_t fixcap = 0xffffffffu) {
  if (fixcap == 0xffffffffu) fixcap = cap;
  SpLayout L{};
  uint64_t o = 0;
  auto take = [&](uint64_t bytes) {
    const uint64_t at = o;
    o = (o + bytes + 255u) & ~255ull;
    return at;
  };
  const uint64_t N1 = (uint64_t)n + 2;
  L.stride = (uint32_t)N1;
  for (int i = 0; i < 26; ++i) L.u32n[i] = take(4 * N1);
  L.fcode = take(4 * (N1 + 1));
  L.ccode = take(4 * (N1 + 1));
  L.pool_owner = take(4 * ((uint64_t)pool + 1));
  L.nw = (n + 63) / 64 + 1;
  L.nsw = (L.nw + 63) / 64 + 1;
  L.stb = take(8ull * L.nw);
  L.sts = take(8ull * L.nsw);
  L.act = take(8ull * L.nw);
  L.acts = take(8ull * L.nsw);
  L.tcb = take(8ull * L.nw);
  L.tcbs = take(8ull * L.nsw);
  L.fcert = take(4 * (m2 + 1));
  L.bcert = take(4 * (m2 + 1));
  L.ccert = take(4 * (m2 + 1));
  L.tc = take(sizeof(SpTc) * N1);
  L.reps = take(4ull * pool * N1);
  L.auts = take(2ull * cap * N1);
  L.ulog_cap = 5 * n + 64;
  L.ulog = take(8ull * L.ulog_cap);
  L.fixcap = fixcap;
  L.fixst = take(8ull * fixcap);
  L.bytes = o;
  return L;
}

// Shared-memory staging: the arrays every refinement step touches (elem,
// pos, in_level, the list of non-singleton cells and the start / active /
// touched-cell bitmaps with their summaries) live in the warp's
// shared-memory region when they fit.
__host__ __device__ inline uint64_t sp_smem_bytes(uint32_t n) {
  const uint64_t nw = (n + 63) / 64 + 1, nsw = (nw + 63) / 64 + 1;
  const uint64_t a = ((uint64_t)n + 2) * 4u;
  return 4 * ((a + 15) & ~15ull) + 3 * 8 * (nw + nsw);
}

struct SpWarp {
  uint32_t *elem, *pos, *inlev, *cnt, *T, *Tc, *cellcnt, *off, *fill, *G, *tmp, *lst1, *lst2;
  uint32_t *seq, *fseq, *bseq, *flabel, *blabel, *dsu, *hist, *pre, *fpos, *bpos, *nsl;
  int32_t *fcode, *ccode, *pool_owner, *pathcode;
  uint32_t *umark;  // per level: undo-log size when the level's child was made
  uint2* ulog;      // undo log: {position | kStartFlag, previous in_level}
  uint2* fixst;     // per stored automorphism: {prefix of seq it fixes, first
                    // position of seq it moves or kNone}, valid for the path
  uint64_t *stb, *sts, *act, *acts, *tcb, *tcbs;
  uint32_t *fcert, *bcert, *ccert, *reps;
  SpTc* tc;
  uint16_t* auts;
  const int32_t* rp;
  const int32_t* col;
  uint32_t n, nw, nsw, stride;  // stride: elements per pool / ring entry
  uint32_t ncells, nact, ntouched, nl1, nl2, npend;
  uint32_t pool_top, pool_cap, aut_cap, max_aut;
  uint32_t utop, ulog_cap, ulog_bad;
  uint32_t fixcap;  // store entries whose fix state is kept (later ones are checked in full)
  // values the serial fold hands to the whole warp
  uint32_t lc, hint;
};

__shared__ SpWarp g_sp[kSpWarps];

// Loads of data that warps on other SMs write during the same launch (the
// shared automorphism store and best leaf of the many-warp search) go
// through L2 only; everything else uses ordinary loads.
template <bool kCg, typename T>
__device__ __forceinline__ T ldx(const T* p) {
  if constexpr (kCg) return __ldcg(p);
  else return *p;
}
__device__ __forceinline__ SpWarp& sp_w() { return g_sp[threadIdx.x >> 5]; }

// ---- bitmaps with a summary word per 64 words ----------------------------
__device__ __forceinline__ bool bm_test(const uint64_t* B, uint32_t p) {
  return (B[p >> 6] >> (p & 63)) & 1ull;
}
// smallest set position >= p, or n
__device__ uint32_t bm_next(const uint64_t* B, const uint64_t* Sm, uint32_t p, uint32_t n,
                            uint32_t nw, uint32_t nsw) {
  if (p >= n) return n;
  uint32_t w = p >> 6;
  const uint64_t x = B[w] & ge_mask(p & 63);
  if (x) return min(n, w * 64 + ctz64(x));
  ++w;
  if (w >= nw) return n;
  uint32_t sw = w >> 6;
  uint64_t y = Sm[sw] & ge_mask(w & 63);
  while (!y) {
    if (++sw >= nsw) return n;
    y = Sm[sw];
  }
  const uint32_t w2 = sw * 64 + ctz64(y);
  if (w2 >= nw) return n;
  return min(n, w2 * 64 + ctz64(B[w2]));
}
// largest set position <= p, or kNone
__device__ uint32_t bm_prev(const uint64_t* B, const uint64_t* Sm, uint32_t p) {
  uint32_t w = p >> 6;
  const uint64_t x = B[w] & low_mask((p & 63) + 1);
  if (x) return w * 64 + msb64(x);
  if (w == 0) return kNone;
  --w;
  uint32_t sw = w >> 6;
  uint64_t y = Sm[sw] & low_mask((w & 63) + 1);
  while (!y) {
    if (sw == 0) return kNone;
    y = Sm[--sw];
  }
  const uint32_t w2 = sw * 64 + msb64(y);
  return w2 * 64 + msb64(B[w2]);
}
// single-writer set / clear (summary kept exact)
__device__ __forceinline__ void bm_set1(uint64_t* B, uint64_t* Sm, uint32_t p) {
  B[p >> 6] |= bit64(p & 63);
  Sm[p >> 12] |= bit64((p >> 6) & 63);
}
__device__ __forceinline__ void bm_clear1(uint64_t* B, uint64_t* Sm, uint32_t p) {
  const uint64_t v = B[p >> 6] & ~bit64(p & 63);
  B[p >> 6] = v;
  if (!v) Sm[p >> 12] &= ~bit64((p >> 6) & 63);
}
__device__ __forceinline__ void bm_set_atomic(uint64_t* B, uint64_t* Sm, uint32_t p) {
  atomicOr((unsigned long long*)&B[p >> 6], (unsigned long long)bit64(p & 63));
  atomicOr((unsigned long long*)&Sm[p >> 12], (unsigned long long)bit64((p >> 6) & 63));
}

// warp: rebuild a summary from its bitmap
__device__ void bm_resummarize(const uint64_t* B, uint64_t* Sm, uint32_t nw, uint32_t nsw) {
  const uint32_t lane = lane_id();
  for (uint32_t sw = 0; sw < nsw; ++sw) {
    const uint32_t w0 = sw * 64 + lane, w1 = w0 + 32;
    const bool a = w0 < nw && B[w0] != 0, b = w1 < nw && B[w1] != 0;
    const uint64_t m = ballot2(a, b);
    if (lane == 0) Sm[sw] = m;
  }
  __syncwarp();
}

__device__ __forceinline__ uint32_t sp_cell_end(const SpWarp& W, uint32_t c) {
  return bm_next(W.stb, W.sts, c + 1, W.n, W.nw, W.nsw);
}
__device__ __forceinline__ uint32_t sp_cell_of(const SpWarp& W, uint32_t p) {
  return bm_prev(W.stb, W.sts, p);
}
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---- undo log of the partition's cell structure ----------------------------
// Every change of a cell start or an in_level after the root refinement is
// logged (by lane 0, in order), so backtracking undoes exactly the changes
// made below the target level instead of rescanning the whole partition.
// Vertex order inside cells is not restored: only cells as sets matter.
constexpr uint32_t kStartFlag = 0x80000000u;

__device__ __forceinline__ void ulog_push(SpWarp& W, uint32_t x, uint32_t old) {
  if (W.utop < W.ulog_cap)
    W.ulog[W.utop++] = make_uint2(x, old);
  else
    W.ulog_bad = 1;  // full: backtracks rescan the partition
}
// lane 0: in_level write / new cell start, logged
__device__ __forceinline__ void set_inlev(SpWarp& W, uint32_t p, uint32_t v) {
  ulog_push(W, p, W.inlev[p]);
  W.inlev[p] = v;
}
__device__ __forceinline__ void add_start(SpWarp& W, uint32_t p) {
  ulog_push(W, p | kStartFlag, 0u);
  bm_set1(W.stb, W.sts, p);
}

// ---------------------------------------------------------------------------
// Rearranging a split cell.  `seg` holds the k touched vertices of the cell
// (cnt[] > 0); they must end up exactly in [r0, r0 + k) -- the neighbour
// fragment for a singleton splitter, the tail for a non-singleton one.
// Touched vertices outside the region swap with untouched vertices inside.
// When `order` is non-null the region is then written in that order.
// ---------------------------------------------------------------------------
__device__ __noinline__ void sp_regroup(const uint32_t* seg, uint32_t k, uint32_t r0,
                                        const uint32_t* order) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  if (lane == 0) W.nl1 = W.nl2 = 0;
  __syncwarp();
  for (uint32_t i = lane; i < k; i += 32) {
    const uint32_t u = seg[i], p = W.pos[u];
    if (p < r0 || p >= r0 + k) W.lst1[atomicAdd(&W.nl1, 1u)] = p;  // touched, misplaced
  }
  for (uint32_t q = r0 + lane; q < r0 + k; q += 32) {
    const uint32_t x = W.elem[q];
    if (W.cnt[x] == 0) W.lst2[atomicAdd(&W.nl2, 1u)] = q;  // hole: untouched inside
  }
  __syncwarp();
  const uint32_t m = W.nl1;  // == nl2
  // read both sides first, then write
  for (uint32_t i0 = 0; i0 < m; i0 += 32) {
    const uint32_t i = i0 + lane;
    uint32_t po = 0, ph = 0, vo = 0, vh = 0;
    if (i < m) {
      po = W.lst1[i];
      ph = W.lst2[i];
      vo = W.elem[po];
      vh = W.elem[ph];
    }
    __syncwarp();
    if (i < m) {
      W.elem[po] = vh;
      W.pos[vh] = po;
      W.elem[ph] = vo;
      W.pos[vo] = ph;
    }
    __syncwarp();
  }
  if (order) {
    for (uint32_t j = lane; j < k; j += 32) {
      const uint32_t u = order[j];
      W.elem[r0 + j] = u;
      W.pos[u] = r0 + j;
    }
  }
  __syncwarp();
}

// Ascending start positions of the non-singleton cells into W.nsl; returns
// their number.  Each lane scans a contiguous range of start-bitmap words and
// an exclusive warp scan places its cells.
__device__ __noinline__ uint32_t sp_list_nonsingleton() {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n, nwr = (n + 63) / 64;
  const uint32_t per = (nwr + 31) / 32;
  const uint32_t w0 = min(nwr, lane * per), w1 = min(nwr, w0 + per);
  const uint64_t lastp = bit64((n - 1) & 63);
  uint32_t cnt = 0;
  for (uint32_t w = w0; w < w1; ++w) {
    const uint64_t b = W.stb[w];
    uint64_t succ = (b >> 1) | ((w + 1 < nwr ? W.stb[w + 1] : 0ull) << 63);
    if (w == nwr - 1) succ |= lastp;
    cnt += popc64(b & ~succ);
  }
  uint32_t off = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(GCL_FULL, off, o);
    if (lane >= (uint32_t)o) off += y;
  }
  const uint32_t total = __shfl_sync(GCL_FULL, off, 31);
  off -= cnt;
  for (uint32_t w = w0; w < w1; ++w) {
    const uint64_t b = W.stb[w];
    uint64_t succ = (b >> 1) | ((w + 1 < nwr ? W.stb[w + 1] : 0ull) << 63);
    if (w == nwr - 1) succ |= lastp;
    uint64_t ns = b & ~succ;
    while (ns) {
      W.nsl[off++] = w * 64 + ctz64(ns);
      ns &= ns - 1;
    }
  }
  __syncwarp();
  return total;
}

// ---------------------------------------------------------------------------
// One refinement step with a non-singleton splitter of at most 32 members
// whose members have at most 32 neighbours in all (partition_refinement.cpp:
// 244-465), warp-synchronously: lane i takes the i-th edge out of the
// splitter; lanes holding the same neighbour are grouped (its count is the
// group's size), the neighbours' leaders are grouped by cell, and each
// touched cell ranks its touched vertices by count with a radix pass over
// ballots.  A cell that splits is rearranged in place: its untouched
// vertices first, then its touched ones in ascending count (the reference's
// fragment order; order inside a fragment is immaterial).  The hash then
// folds every non-singleton cell in position order -- an untouched one
// contributes its start, a touched one its fragments -- and lane 0 does the
// bookkeeping of the splits (starts, in_level, active set, hint) in the same
// order.  Nothing goes through the per-step scratch arrays of the general
// path.  Returns false, having changed nothing, when the splitter is too
// large; `lc` and `hint` are the refinement's running hash and hint.
// ---------------------------------------------------------------------------
__device__ __noinline__ bool sp_refine_small(uint32_t s, uint32_t len, uint32_t lvl1,
                                             uint32_t* lc_io, uint32_t* hint_io) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  if (len > 32) return false;
  // the splitter's edges, lane by lane
  uint32_t d = 0;
  int32_t b = 0;
  if (lane < len) {
    const uint32_t w = W.elem[s + lane];
    b = W.rp[w];
    d = (uint32_t)(W.rp[w + 1] - b);
  }
  uint32_t incl = d;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(GCL_FULL, incl, o);
    if (lane >= (uint32_t)o) incl += y;
  }
  const uint32_t D = __shfl_sync(GCL_FULL, incl, 31);
  if (D > 32) return false;
  const uint32_t excl = incl - d;
  const uint32_t nonempty = __ballot_sync(GCL_FULL, d > 0);
  const uint32_t firsts = __reduce_or_sync(GCL_FULL, d > 0 ? (1u << excl) : 0u);
  uint32_t u = kNone;
  {
    // lane i < D: member = the k-th non-empty one, k = firsts up to lane i
    const uint32_t k = (uint32_t)__popc(firsts & (lanemask_lt() | (1u << lane)));
    const int src = lane < D ? __fns(nonempty, 0, (int)k) : 0;
    const int32_t bs = __shfl_sync(GCL_FULL, b, src);
    const uint32_t es = __shfl_sync(GCL_FULL, excl, src);
    if (lane < D) u = (uint32_t)W.col[bs + (int32_t)(lane - es)];
  }
  // the neighbour's cell; singleton cells never split (:257-259)
  uint32_t p = 0, c = kNone, L = 0;
  if (u != kNone) {
    p = W.pos[u];
    c = sp_cell_of(W, p);
    L = sp_cell_end(W, c) - c;
    if (L <= 1) u = kNone;
  }
  const uint32_t gu = __match_any_sync(GCL_FULL, u);
  const uint32_t cnt = (uint32_t)__popc(gu);  // u's neighbours in the splitter
  const bool lead = u != kNone && lane == (uint32_t)(__ffs(gu) - 1);
  const uint32_t gc = __match_any_sync(GCL_FULL, lead ? c : kNone);
  const uint32_t k = lead ? (uint32_t)__popc(gc) : 0u;  // touched vertices of the cell
  // rank by count within the cell (radix pass, counts <= 32: 6 bits)
  uint32_t peers = lead ? gc : 0u, less = 0;
  for (int bit = 5; bit >= 0; --bit) {
    const bool one = (cnt >> bit) & 1u;
    const uint32_t m1 = __ballot_sync(GCL_FULL, lead && one);
    if (lead) {
      if (one) {
        less += (uint32_t)__popc(peers & ~m1);
        peers &= m1;
      } else {
        peers &= ~m1;
      }
    }
  }
  const uint32_t eqidx = (uint32_t)__popc(peers & lanemask_lt());
  const uint32_t fsize = (uint32_t)__popc(peers);
  const bool uniform = lead && k == L && fsize == k;  // one common count: no split
  const bool split = lead && !uniform;
  const uint32_t R0 = c + (L - k);
  const uint32_t f = R0 + less;  // this vertex's fragment start
  const bool cell_lead = lead && lane == (uint32_t)(__ffs(gc) - 1);
  // rearrange the split cells: touched vertices to R0 + rank, the untouched
  // vertices found in [R0, c + L) to the positions the touched ones leave
  uint32_t x = 0, h = 0;
  bool out = false;
  if (split) {
    const bool in = p >= R0;
    const uint32_t inner = __reduce_or_sync(gc, in ? (1u << (p - R0)) : 0u);
    const uint32_t outs = __ballot_sync(gc, !in);
    if (!in) {
      const uint32_t j = (uint32_t)__popc(outs & lanemask_lt());
      const uint32_t holes = ~inner & (k >= 32 ? 0xffffffffu : ((1u << k) - 1u));
      h = R0 + (uint32_t)__fns(holes, 0, (int)j + 1);
      x = W.elem[h];
      out = true;
    }
  }
  __syncwarp();
  if (out) {
    W.elem[p] = x;
    W.pos[x] = p;
  }
  if (split) {
    const uint32_t t = f + eqidx;
    W.elem[t] = u;
    W.pos[u] = t;
  }
  if (cell_lead) bm_set_atomic(W.tcb, W.tcbs, c);
  __syncwarp();
  // the fold over the non-singleton cells in position order (:253-465)
  uint32_t lc = *lc_io, hint = *hint_io;
  const uint32_t K = sp_list_nonsingleton();
  uint32_t pend = 0;  // lanes whose fragment is a new cell start
  for (uint32_t i0 = 0; i0 < K; i0 += 32) {
    const uint32_t il = i0 + lane;
    const uint32_t cl = il < K ? W.nsl[il] : 0u;
    const uint32_t tmask = __ballot_sync(GCL_FULL, il < K && bm_test(W.tcb, cl));
    const uint32_t cnt32 = min(32u, K - i0);
    if (!tmask) {  // 32 untouched cells: each member has count 0, item = start
      lc = mash_fold32(lc, cl, cnt32);
      continue;
    }
    for (uint32_t jj = 0; jj < cnt32; ++jj) {
      const uint32_t cc = __shfl_sync(GCL_FULL, cl, (int)jj);
      if (!((tmask >> jj) & 1u)) {
        lc = mash(lc, cc);  // untouched: every member has count 0
        continue;
      }
      const uint32_t src = (uint32_t)__ffs(__ballot_sync(GCL_FULL, cell_lead && c == cc)) - 1;
      const bool uni = __shfl_sync(GCL_FULL, uniform, (int)src);
      if (uni) {
        lc = mash(lc, __shfl_sync(GCL_FULL, cnt, (int)src) + cc);
        continue;
      }
      const uint32_t Lc = __shfl_sync(GCL_FULL, L, (int)src);
      const uint32_t kc = __shfl_sync(GCL_FULL, k, (int)src);
      const bool was = bm_test(W.act, cc);
      const uint32_t oldlev = W.inlev[cc];
      __syncwarp();
      uint32_t maxsz = 0, maxf = cc, lastf = cc;
      if (Lc > kc) {  // the untouched fragment first
        lc = mash(lc, 0u + cc);
        if (lane == 0) set_inlev(W, cc, lvl1);
        maxsz = Lc - kc;
      }
      // the touched fragments in ascending count (= ascending start)
      uint32_t F = __ballot_sync(GCL_FULL, split && c == cc && eqidx == 0);
      while (F) {
        const uint32_t fm = __reduce_min_sync(GCL_FULL, ((F >> lane) & 1u) ? f : kNone);
        const uint32_t s2 = (uint32_t)__ffs(__ballot_sync(GCL_FULL, ((F >> lane) & 1u) && f == fm)) - 1;
        F &= ~(1u << s2);
        const uint32_t sz = __shfl_sync(GCL_FULL, fsize, (int)s2);
        lc = mash(lc, __shfl_sync(GCL_FULL, cnt, (int)s2) + fm);
        if (fm != cc) {
          pend |= 1u << s2;
          if (sz == 1) hint = fm;
        }
        if (lane == 0) {
          set_inlev(W, fm, lvl1);
          if (fm != cc) {
            W.ncells += 1;
            if (!bm_test(W.act, fm)) {
              bm_set1(W.act, W.acts, fm);
              W.nact += 1;
            }
          }
        }
        if (sz > maxsz) {
          maxsz = sz;
          maxf = fm;
        }
        lastf = fm;
      }
      if (lane == 0) {
        if (!was) {
          if (!bm_test(W.act, cc)) {
            bm_set1(W.act, W.acts, cc);
            W.nact += 1;
          }
          if (bm_test(W.act, maxf)) {
            bm_clear1(W.act, W.acts, maxf);
            W.nact -= 1;
          }
        }
        set_inlev(W, lastf, oldlev);
      }
      __syncwarp();
    }
  }
  // the new starts, set after the fold (which walked the old ones)
  while (pend) {
    const uint32_t s2 = (uint32_t)__ffs(pend) - 1;
    pend &= pend - 1;
    const uint32_t fs = __shfl_sync(GCL_FULL, f, (int)s2);
    if (lane == 0) add_start(W, fs);
  }
  if (cell_lead) {  // the touched-cell marks go
    W.tcb[c >> 6] = 0;
    W.tcbs[c >> 12] = 0;
  }
  __syncwarp();
  *lc_io = lc;
  *hint_io = hint;
  return true;
}

// ---------------------------------------------------------------------------
// Partition_s_refinement (partition_refinement.cpp:150-485).  The active
// bitmap holds the initially active cells; returns the code (-1 on a failed
// consistency check).  The caller increments the level.
// ---------------------------------------------------------------------------
__device__ __noinline__ int sp_refine(uint32_t level) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n, nw = W.nw, nsw = W.nsw;
  const uint32_t lvl1 = level + 1;
  uint32_t lc = W.ncells, hint = 0;
  uint64_t iters = 0;
  int ok = 1;
  // the arrays a step touches, in registers for the whole refinement (the
  // warp record's pointers would otherwise be reloaded after every store)
  uint32_t* const elem = W.elem;
  uint32_t* const pos = W.pos;
  uint64_t* const stb = W.stb;
  uint64_t* const sts = W.sts;
  uint64_t* const act = W.act;
  uint64_t* const acts = W.acts;
  const int32_t* const rp = W.rp;
  const int32_t* const col = W.col;
  uint32_t* const inlev = W.inlev;
  uint2* const ulog = W.ulog;
  const uint32_t ucap = W.ulog_cap;
  // the cell and active counts and the undo log's top, kept by every lane
  // alike during the singleton steps; the warp record holds them while the
  // other paths run (they update them there) and after the refinement
  uint32_t ncells = W.ncells, nact = W.nact, utop = W.utop;
  while (ncells < n && nact > 0) {
    if (++iters > 4ull * n + 64) {  // every step removes an active cell or splits one
      ok = 0;
      break;
    }
    uint32_t s;
    if (bm_test(act, hint)) {
      s = hint;
    } else {
      s = bm_next(act, acts, hint + 1, n, nw, nsw);
      if (s >= n) s = bm_next(act, acts, 0, n, nw, nsw);
    }
    if (s >= n) {
      ok = 0;
      break;
    }
    __syncwarp();
    if (lane == 0) bm_clear1(act, acts, s);
    nact -= 1;
    const uint32_t e = bm_test(stb, s + 1) || s + 1 >= n ? s + 1
                                                          : bm_next(stb, sts, s + 1, n, nw, nsw);
    const uint32_t len = e - s;
    lc = mash(lc, s + e - 1);
    if (len > 1) lc = mash(lc, len);

    // Singleton splitter {w} with at most 32 neighbours: lane i holds
    // neighbour i; lanes whose neighbours share a (non-singleton) cell are
    // grouped with match_any; a cell that is not all neighbours splits into
    // [neighbours, non-neighbours]: its misplaced neighbours swap with the
    // non-neighbours inside its first k positions, then the split cells are
    // folded in position order (:296-309, 399-435).
    int32_t sb = 0, sd = 0;
    if (len == 1) {
      const uint32_t w = elem[s];
      sb = rp[w];
      sd = rp[w + 1] - sb;
    }
    if (len == 1 && sd <= 32) {
      const bool have = (int32_t)lane < sd;
      uint32_t u = 0, p = 0, c = kNone, L = 0;
      if (have) {
        u = (uint32_t)col[sb + (int32_t)lane];
        p = pos[u];
        c = bm_prev(stb, sts, p);
        L = bm_next(stb, sts, c + 1, n, nw, nsw) - c;
      }
      const bool act_l = have && L > 1;
      const uint32_t grp = __match_any_sync(GCL_FULL, act_l ? c : kNone);
      const uint32_t k = (uint32_t)__popc(grp);
      const bool spl_l = act_l && k < L;
      uint32_t h = 0, x = 0;
      bool mv = false;
      if (spl_l) {
        const bool in = p < c + k;
        const uint32_t inner = __reduce_or_sync(grp, in ? (1u << (p - c)) : 0u);
        const uint32_t outs = __ballot_sync(grp, !in);
        if (!in) {
          const uint32_t j = (uint32_t)__popc(outs & lanemask_lt());
          const uint32_t holes = ~inner & (k >= 32 ? 0xffffffffu : ((1u << k) - 1u));
          h = c + (uint32_t)__fns(holes, 0, (int)j + 1);
          x = elem[h];
          mv = true;
        }
      }
      // whether each split cell was active, read before any of this step's
      // active-set writes (they only touch the split cells' own starts)
      const bool lead = spl_l && lane == (uint32_t)(__ffs(grp) - 1);
      const bool was_l = lead && bm_test(act, c);
      __syncwarp();
      if (mv) {
        elem[h] = u;
        pos[u] = h;
        elem[p] = x;
        pos[x] = p;
      }
      // split cells in position order: hash, in_level, starts, active set;
      // hint and hash are the same on every lane, lane 0 writes
      uint32_t leaders = __ballot_sync(GCL_FULL, lead);
      while (leaders) {
        const bool mine = (leaders >> lane) & 1u;
        const uint32_t cmin = __reduce_min_sync(GCL_FULL, mine ? c : kNone);
        const uint32_t src = (uint32_t)__ffs(__ballot_sync(GCL_FULL, mine && c == cmin)) - 1;
        const uint32_t kk = __shfl_sync(GCL_FULL, k, (int)src);
        const uint32_t LL = __shfl_sync(GCL_FULL, L, (int)src);
        const bool was = __shfl_sync(GCL_FULL, was_l, (int)src);
        leaders &= ~(1u << src);
        const uint32_t pp = cmin + kk;
        lc = mash(lc, pp - 1);  // cell.first + neighbors_size - 1
        const uint32_t nb = kk, nn = LL - kk;
        const bool to_rest = was || nb >= nn;
        if (to_rest) {
          if (nn == 1) hint = pp;
        } else {
          if (nb == 1) hint = cmin;
        }
        if (lane == 0) {
          // in_level of both fragments and the new start, logged in the
          // order set_inlev / add_start would log them
          const uint32_t oldc = inlev[cmin], oldp = inlev[pp];
          if (utop + 3 <= ucap) {
            ulog[utop] = make_uint2(pp, oldp);
            ulog[utop + 1] = make_uint2(cmin, oldc);
            ulog[utop + 2] = make_uint2(pp | kStartFlag, 0u);
          } else {
            W.ulog_bad = 1;  // full: backtracks rescan the partition
          }
          inlev[pp] = oldc;
          inlev[cmin] = lvl1;
          bm_set1(stb, sts, pp);
          bm_set1(act, acts, to_rest ? pp : cmin);
        }
        if (utop + 3 <= ucap) utop += 3;
        ncells += 1;
        nact += 1;
      }
      __syncwarp();
      continue;
    }
    // the other paths keep the counts in the warp record
    if (lane == 0) {
      W.ncells = ncells;
      W.nact = nact;
      W.utop = utop;
      W.ntouched = 0;
    }
    __syncwarp();

    // a small non-singleton splitter: warp-synchronous, no scratch arrays
    if (len > 1 && sp_refine_small(s, len, lvl1, &lc, &hint)) {
      ncells = W.ncells;
      nact = W.nact;
      utop = W.utop;
      continue;
    }

    // count neighbours in the splitter, record touched vertices and cells
    // (cells that are singletons never split and are skipped, :257-259)
    if (len == 1) {
      const uint32_t w = W.elem[s];
      const int32_t b = W.rp[w], d = W.rp[w + 1] - b;
      for (int32_t i = (int32_t)lane; i < d; i += 32) {
        const uint32_t u = (uint32_t)W.col[b + i];
        const uint32_t c = sp_cell_of(W, W.pos[u]);
        if (sp_cell_end(W, c) - c == 1) continue;
        if (atomicAdd(&W.cnt[u], 1u) == 0) {
          const uint32_t t = atomicAdd(&W.ntouched, 1u);
          W.T[t] = u;
          W.Tc[t] = c;
          if (atomicAdd(&W.cellcnt[c], 1u) == 0) bm_set_atomic(W.tcb, W.tcbs, c);
        }
      }
    } else {
      for (uint32_t q = s + lane; q < e; q += 32) {
        const uint32_t w = W.elem[q];
        const int32_t b = W.rp[w], f = W.rp[w + 1];
        for (int32_t i = b; i < f; ++i) {
          const uint32_t u = (uint32_t)W.col[i];
          const uint32_t c = sp_cell_of(W, W.pos[u]);
          if (sp_cell_end(W, c) - c == 1) continue;
          if (atomicAdd(&W.cnt[u], 1u) == 0) {
            const uint32_t t = atomicAdd(&W.ntouched, 1u);
            W.T[t] = u;
            W.Tc[t] = c;
            if (atomicAdd(&W.cellcnt[c], 1u) == 0) bm_set_atomic(W.tcb, W.tcbs, c);
          }
        }
      }
    }
    __syncwarp();
    const uint32_t nt = W.ntouched;
    // group the touched vertices by cell (counting sort, cells in order)
    {
      uint32_t run = 0;
      uint32_t c = bm_next(W.tcb, W.tcbs, 0, n, nw, nsw);
      while (c < n) {
        const uint32_t k = W.cellcnt[c];
        if (lane == 0) W.off[c] = run;
        run += k;
        c = bm_next(W.tcb, W.tcbs, c + 1, n, nw, nsw);
      }
      __syncwarp();
      for (uint32_t i = lane; i < nt; i += 32) {
        const uint32_t c2 = W.Tc[i];
        W.G[W.off[c2] + atomicAdd(&W.fill[c2], 1u)] = W.T[i];
      }
      __syncwarp();
    }

    if (len == 1) {
      // every touched cell that is not all neighbours splits into
      // [neighbours, non-neighbours] (:296-309, 399-435)
      uint32_t c = bm_next(W.tcb, W.tcbs, 0, n, nw, nsw);
      while (c < n) {
        const uint32_t k = W.cellcnt[c], ce = sp_cell_end(W, c), L = ce - c;
        const uint32_t cnext = bm_next(W.tcb, W.tcbs, c + 1, n, nw, nsw);
        if (k < L) {
          sp_regroup(W.G + W.off[c], k, c, nullptr);
          const uint32_t p = c + k;
          lc = mash(lc, p - 1);
          const bool was = bm_test(W.act, c);
          if (lane == 0) {
            set_inlev(W, p, W.inlev[c]);
            set_inlev(W, c, lvl1);
            add_start(W, p);
            W.ncells += 1;
            const uint32_t nb = k, nn = L - k;
            if (was || nb >= nn) {
              bm_set1(W.act, W.acts, p);
              W.nact += 1;
              if (nn == 1) hint = p;
            } else {
              if (!was) {
                bm_set1(W.act, W.acts, c);
                W.nact += 1;
              }
              if (nb == 1) hint = c;
            }
            W.hint = hint;
          }
          __syncwarp();
          hint = W.hint;
        }
        c = cnext;
      }
    } else {
      // every non-singleton cell in order: common count, or fragments in
      // ascending count with the untouched (count 0) fragment first.  Cells
      // are taken 32 at a time; untouched ones only hash their start.
      const uint32_t K = sp_list_nonsingleton();
      for (uint32_t i0 = 0; i0 < K; i0 += 32) {
        const uint32_t il = i0 + lane;
        const uint32_t cl = il < K ? W.nsl[il] : 0u;
        const uint32_t tmask = __ballot_sync(GCL_FULL, il < K && bm_test(W.tcb, cl));
        const uint32_t cnt32 = min(32u, K - i0);
        if (!tmask) {  // 32 untouched cells: item = start
          lc = mash_fold32(lc, cl, cnt32);
          continue;
        }
        for (uint32_t jj = 0; jj < cnt32; ++jj) {
          const uint32_t c = __shfl_sync(GCL_FULL, cl, (int)jj);
          if (!((tmask >> jj) & 1u)) {
            lc = mash(lc, c);  // every member has count 0
            continue;
          }
          const uint32_t ce = sp_cell_end(W, c), L = ce - c;
          const uint32_t k = W.cellcnt[c];
          const uint32_t* seg = W.G + W.off[c];
          uint32_t mn = 0xffffffffu, mx = 0;
          for (uint32_t i = lane; i < k; i += 32) {
            const uint32_t x = W.cnt[seg[i]];
            mn = min(mn, x);
            mx = max(mx, x);
          }
          mn = __reduce_min_sync(GCL_FULL, mn);
          mx = __reduce_max_sync(GCL_FULL, mx);
          if (k == L && mn == mx) {
            lc = mash(lc, mn + c);
            continue;
          }
          // counting sort of the touched vertices by count
          const uint32_t range = mx - mn + 1;
          for (uint32_t i = lane; i < range; i += 32) W.hist[i] = 0;
          __syncwarp();
          for (uint32_t i = lane; i < k; i += 32) atomicAdd(&W.hist[W.cnt[seg[i]] - mn], 1u);
          __syncwarp();
          if (lane == 0) {
            uint32_t run = 0;
            for (uint32_t i = 0; i < range; ++i) {
              W.pre[i] = run;
              run += W.hist[i];
            }
          }
          __syncwarp();
          for (uint32_t i = lane; i < k; i += 32) {
            const uint32_t u = seg[i];
            const uint32_t d = W.cnt[u] - mn;
            W.tmp[atomicAdd(&W.pre[d], 1u)] = u;  // pre[d] ends at the fragment end
          }
          __syncwarp();
          const uint32_t r0 = c + (L - k);
          sp_regroup(seg, k, r0, W.tmp);
          // fragments: hash, starts, in_level, active (:326-465)
          const bool was = bm_test(W.act, c);
          const uint32_t oldlev = W.inlev[c];
          __syncwarp();
          if (lane == 0) {
            uint32_t maxsz = 0, maxf = c, lastf = c, nfr = 0;
            if (L > k) {  // untouched fragment first
              lc = mash(lc, 0u + c);
              set_inlev(W, c, lvl1);
              maxsz = L - k;
              nfr = 1;
            }
            uint32_t f = r0;
            for (uint32_t i = 0; i < range; ++i) {
              const uint32_t sz = W.hist[i];
              if (!sz) continue;
              lc = mash(lc, mn + i + f);
              set_inlev(W, f, lvl1);
              if (f != c) {
                W.fpos[W.npend++] = f;  // set after the fold: the fold walks the old starts
                W.ncells += 1;
                if (!bm_test(W.act, f)) {
                  bm_set1(W.act, W.acts, f);
                  W.nact += 1;
                }
                if (sz == 1) hint = f;
              }
              if (sz > maxsz) {
                maxsz = sz;
                maxf = f;
              }
              lastf = f;
              f += sz;
              ++nfr;
            }
            if (!was) {
              if (!bm_test(W.act, c)) {
                bm_set1(W.act, W.acts, c);
                W.nact += 1;
              }
              if (bm_test(W.act, maxf)) {
                bm_clear1(W.act, W.acts, maxf);
                W.nact -= 1;
              }
            }
            set_inlev(W, lastf, oldlev);
            W.lc = lc;
            W.hint = hint;
          }
          __syncwarp();
          lc = W.lc;
          hint = W.hint;
        }
      }
    }
    // new starts of the non-singleton fold
    __syncwarp();
    if (lane == 0) {
      for (uint32_t i = 0; i < W.npend; ++i) add_start(W, W.fpos[i]);
      W.npend = 0;
    }
    // reset per-step scratch
    __syncwarp();
    for (uint32_t i = lane; i < nt; i += 32) {
      const uint32_t u = W.T[i], c = W.Tc[i];
      W.cnt[u] = 0;
      W.cellcnt[c] = 0;
      W.fill[c] = 0;
      W.tcb[c >> 6] = 0;
      W.tcbs[c >> 12] = 0;
    }
    __syncwarp();
    ncells = W.ncells;
    nact = W.nact;
    utop = W.utop;
  }
  if (lane == 0) {
    W.ncells = ncells;
    W.utop = utop;
  }
  // clear what is left of the active set
  __syncwarp();
  for (uint32_t w = lane; w < nw; w += 32) W.act[w] = 0;
  for (uint32_t w = lane; w < nsw; w += 32) W.acts[w] = 0;
  if (lane == 0) W.nact = 0;
  __syncwarp();
  if (!ok) return -1;
  return cleanup(mash(lc, W.ncells));
}

// split_by_and_refine's split (partition_refinement.cpp:486-528)
__device__ __forceinline__ bool sp_individualize(uint32_t level, uint32_t v, uint32_t t) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t e = sp_cell_end(W, t);
  if (e - t <= 1) return false;
  __syncwarp();
  if (lane == 0) {
    W.umark[level] = W.utop;  // backtracking to `level` undoes from here
    const uint32_t p = W.pos[v], x = W.elem[t];
    W.elem[p] = x;
    W.pos[x] = p;
    W.elem[t] = v;
    W.pos[v] = t;
    add_start(W, t + 1);
    W.ncells += 1;
    set_inlev(W, t + 1, W.inlev[t]);
    set_inlev(W, t, level + 1);
    bm_set1(W.act, W.acts, t);
    W.nact = 1;
  }
  __syncwarp();
  return true;
}

// reconstruct_at_level (partition_refinement.cpp:541-604): a start survives
// unless the cell before it was created after level Lv; a surviving start
// whose own cell is that new takes the in_level of the first following cell
// created at or before Lv.  Each lane handles a contiguous range of words;
// prefix max / suffix min scans carry the neighbouring starts across lanes.
__device__ __noinline__ bool sp_backtrack(uint32_t Lv) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n, nw = (n + 63) / 64;
  const uint32_t per = (nw + 31) / 32;
  const uint32_t w0 = min(nw, lane * per), w1 = min(nw, w0 + per);
  // chunk summary: last start (and whether it is "big"), first non-big start
  uint32_t last = kNone, firstsmall = kNone;
  bool lastbig = false;
  for (uint32_t w = w0; w < w1; ++w) {
    uint64_t b = W.stb[w];
    while (b) {
      const uint32_t p = w * 64 + ctz64(b);
      b &= b - 1;
      const bool big = W.inlev[p] > Lv;
      last = p;
      lastbig = big;
      if (!big && firstsmall == kNone) firstsmall = p;
    }
  }
  // previous start before this chunk: max over lower lanes of `last`
  uint32_t prev_last = kNone;
  bool prev_big = false;
  {
    // encode (position+1) so kNone sorts lowest
    uint32_t key = last == kNone ? 0u : last + 1;
    uint32_t bigbit = lastbig ? 1u : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t k2 = __shfl_up_sync(GCL_FULL, key, o);
      const uint32_t b2 = __shfl_up_sync(GCL_FULL, bigbit, o);
      if (lane >= (uint32_t)o && k2 > key) {
        key = k2;
        bigbit = b2;
      }
    }
    // exclusive: take the inclusive value of lane-1
    const uint32_t kx = __shfl_up_sync(GCL_FULL, key, 1);
    const uint32_t bx = __shfl_up_sync(GCL_FULL, bigbit, 1);
    if (lane > 0 && kx) {
      prev_last = kx - 1;
      prev_big = bx != 0;
    }
  }
  // first non-big start after this chunk: min over higher lanes
  uint32_t next_small = kNone;
  {
    uint32_t key = firstsmall;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t k2 = __shfl_down_sync(GCL_FULL, key, o);
      if (lane + (uint32_t)o < 32 && k2 < key) key = k2;
    }
    const uint32_t kx = __shfl_down_sync(GCL_FULL, key, 1);
    if (lane < 31) next_small = kx;
  }
  // decide survivors and new in_levels; remember the writes
  bool bad = false;
  __syncwarp();
  {
    bool pbig = prev_big;
    const bool have_prev = prev_last != kNone;
    bool first_in_chunk = true;
    // the new in_level of a surviving big start: first non-big start after it
    for (uint32_t w = w0; w < w1; ++w) {
      uint64_t b = W.stb[w];
      uint64_t keep = b;
      uint64_t bb = b;
      while (bb) {
        const uint32_t p = w * 64 + ctz64(bb);
        bb &= bb - 1;
        const bool big = W.inlev[p] > Lv;
        const bool has_prev = !first_in_chunk || have_prev;
        const bool survive = !(has_prev && pbig);
        if (!survive) keep &= ~bit64(p & 63);
        if (survive && big) {
          // closing cell: next non-big start after p
          uint32_t j = kNone;
          uint64_t rest = bb;
          uint32_t ww = w;
          while (true) {
            while (rest) {
              const uint32_t q = ww * 64 + ctz64(rest);
              rest &= rest - 1;
              if (W.inlev[q] <= Lv) {
                j = q;
                break;
              }
            }
            if (j != kNone) break;
            if (++ww >= w1) break;
            rest = W.stb[ww];
          }
          if (j == kNone) j = next_small;
          if (j == kNone) {
            bad = true;
          } else {
            W.tmp[p] = W.inlev[j];  // staged new in_level
          }
        }
        pbig = big;
        first_in_chunk = false;
      }
      W.lst1[w] = (uint32_t)keep;          // staged word (low half)
      W.lst2[w] = (uint32_t)(keep >> 32);  // staged word (high half)
    }
  }
  if (__any_sync(GCL_FULL, bad)) return false;
  __syncwarp();
  // apply: in_levels of surviving big starts, then the start words
  uint32_t removed = 0;
  for (uint32_t w = w0; w < w1; ++w) {
    const uint64_t old = W.stb[w];
    const uint64_t keep = ((uint64_t)W.lst2[w] << 32) | W.lst1[w];
    uint64_t sb = keep;
    while (sb) {
      const uint32_t p = w * 64 + ctz64(sb);
      sb &= sb - 1;
      if (W.inlev[p] > Lv) W.inlev[p] = W.tmp[p];
    }
    removed += popc64(old) - popc64(keep);
    W.stb[w] = keep;
  }
  removed = __reduce_add_sync(GCL_FULL, removed);
  __syncwarp();
  bm_resummarize(W.stb, W.sts, nw, W.nsw);
  if (lane == 0) W.ncells -= removed;
  __syncwarp();
  return true;
}

// Backtrack to node level Lv by undoing the logged changes made since that
// node's child was created: the same cells as reconstruct_at_level.  Every
// start created below Lv is cleared, and every in_level changed below Lv
// returns to the value before its first change (entries are processed in
// parallel: per position the earliest entry wins).
__device__ __forceinline__ bool sp_backtrack_log(uint32_t Lv) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  if (W.ulog_bad) {
    const bool ok = sp_backtrack(Lv);
    __syncwarp();
    return ok;
  }
  const uint32_t lo = W.umark[Lv], hi = W.utop;
  if (lo > hi) return false;
  for (uint32_t i = lo + lane; i < hi; i += 32) {
    const uint2 e = W.ulog[i];
    if (!(e.x & kStartFlag)) W.tmp[e.x] = 0xffffffffu;
  }
  __syncwarp();
  for (uint32_t i = lo + lane; i < hi; i += 32) {
    const uint2 e = W.ulog[i];
    if (!(e.x & kStartFlag)) atomicMin(&W.tmp[e.x], i);
  }
  __syncwarp();
  uint32_t removed = 0;
  for (uint32_t i = lo + lane; i < hi; i += 32) {
    const uint2 e = W.ulog[i];
    if (e.x & kStartFlag) {
      const uint32_t p = e.x & ~kStartFlag;
      atomicAnd((unsigned long long*)&W.stb[p >> 6], (unsigned long long)~bit64(p & 63));
      ++removed;
    } else if (W.tmp[e.x] == i) {
      W.inlev[e.x] = e.y;
    }
  }
  __syncwarp();
  for (uint32_t i = lo + lane; i < hi; i += 32) {
    const uint2 e = W.ulog[i];
    if (e.x & kStartFlag) {
      const uint32_t w = (e.x & ~kStartFlag) >> 6;
      if (W.stb[w] == 0)
        atomicAnd((unsigned long long*)&W.sts[w >> 6], (unsigned long long)~bit64(w & 63));
    }
  }
  removed = __reduce_add_sync(GCL_FULL, removed);
  __syncwarp();
  if (lane == 0) {
    W.ncells -= removed;
    W.utop = lo;
  }
  __syncwarp();
  return true;
}

// ---- leaves ----------------------------------------------------------------
// Certificate of a discrete partition: for every vertex, the canonical
// positions of its neighbours in ascending order, stored at its CSR offset.
__device__ __forceinline__ void sp_leaf_cert(uint32_t* cert) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  for (uint32_t v = lane; v < W.n; v += 32) {
    const int32_t b = W.rp[v], e = W.rp[v + 1];
    for (int32_t i = b; i < e; ++i) {
      const uint32_t x = W.pos[W.col[i]];
      int32_t j = i - 1;
      while (j >= b && cert[j] > x) {  // insertion sort (rows are short)
        cert[j + 1] = cert[j];
        --j;
      }
      cert[j + 1] = x;
    }
  }
  __syncwarp();
}

// Compare the certificate rows of the current leaf (vertex order elem[])
// with a stored leaf (vertex order label[], rows in cert2) in canonical
// row order.  upper: compare_adj_upper (entries right of the diagonal,
// sequential.cpp:114-124); otherwise full-row equality.  Returns -1/0/+1.
template <bool kCg = false>
__device__ __forceinline__ int sp_cmp_leaf(const uint32_t* cur, const uint32_t* label,
                                        const uint32_t* cert2, bool upper) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n;
  for (uint32_t i0 = 0; i0 < n; i0 += 32) {
    const uint32_t i = i0 + lane;
    int r = 0;
    if (i < n) {
      const uint32_t va = W.elem[i], vb = ldx<kCg>(label + i);
      int32_t a = W.rp[va], ae = W.rp[va + 1], b = W.rp[vb], be = W.rp[vb + 1];
      if (upper) {
        while (a < ae && cur[a] <= i) ++a;
        while (b < be && ldx<kCg>(cert2 + b) <= i) ++b;
      }
      while (true) {
        const bool ea = a >= ae, eb = b >= be;
        if (ea && eb) break;
        if (ea) {  // b has a 1 where a has 0
          r = -1;
          break;
        }
        if (eb) {
          r = 1;
          break;
        }
        const uint32_t x = cur[a], y = ldx<kCg>(cert2 + b);
        if (x != y) {
          r = x < y ? 1 : -1;
          break;
        }
        ++a;
        ++b;
      }
    }
    const uint32_t diff = __ballot_sync(GCL_FULL, r != 0);
    if (diff) {
      const int src = __ffs(diff) - 1;
      return __shfl_sync(GCL_FULL, r, src);
    }
  }
  return 0;
}

__device__ __forceinline__ void sp_copy_u32(uint32_t* dst, const uint32_t* src, uint32_t k) {
  const uint32_t lane = lane_id();
  for (uint32_t i = lane; i < k; i += 32) dst[i] = src[i];
  __syncwarp();
}

// get_gca_level (sequential.cpp:183-213)
__device__ __forceinline__ int sp_gca(const uint32_t* a, uint32_t na, uint32_t seqlen) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t m = min(na, seqlen);
  for (uint32_t j0 = 0; j0 < m; j0 += 32) {
    const uint32_t j = j0 + lane;
    const uint32_t b = __ballot_sync(GCL_FULL, j < m && a[j] != W.seq[j]);
    if (b) return (int)(j0 + (uint32_t)(__ffs(b) - 1)) + 1;
  }
  return -1;
}

// first non-singleton cell (target_cell_selector, partition_refinement.cpp:607-655)
__device__ __forceinline__ uint32_t sp_first_nonsingleton() {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n, nw = (n + 63) / 64;
  for (uint32_t w0 = 0; w0 < nw; w0 += 32) {
    const uint32_t w = w0 + lane;
    uint64_t ns = 0;
    if (w < nw) {
      const uint64_t b = W.stb[w];
      const uint64_t nb = (w + 1 < nw) ? W.stb[w + 1] : 0ull;
      uint64_t succ = (b >> 1) | (nb << 63);  // bit p set: p+1 is a start
      const uint32_t lastp = n - 1;
      if ((lastp >> 6) == w) succ |= bit64(lastp & 63);  // the last position ends its cell
      ns = b & ~succ;
    }
    const uint32_t bal = __ballot_sync(GCL_FULL, ns != 0);
    if (bal) {
      const int src = __ffs(bal) - 1;
      const uint32_t p = (uint32_t)src + w0;
      const uint64_t x = bcast64(ns, src);
      return p * 64 + ctz64(x);
    }
  }
  return kNone;
}

// next representative of target cell idx: smallest vertex >= counter among
// its members whose representative is itself (sequential.cpp:359-361)
__device__ __forceinline__ uint32_t sp_next_rep(const SpTc& t) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t* reps = t.rslot >= 0 ? W.reps + (uint64_t)t.rslot * W.stride : nullptr;
  uint32_t best = kNone;
  for (uint32_t q = t.first + lane; q < t.first + t.len; q += 32) {
    const uint32_t v = W.elem[q];
    if (v >= t.counter && v < best && (!reps || reps[v] == v)) best = v;
  }
  return __reduce_min_sync(GCL_FULL, best);
}

__device__ __forceinline__ uint32_t sp_find(volatile uint32_t* d, uint32_t x, uint32_t n) {
  uint32_t p = d[x];
  for (uint32_t step = 0; p < x && step <= n; ++step) {
    x = p;
    p = d[x];
  }
  return x;
}

// Merge the cycles of permutation pm on the `count` vertices members[] into
// the min-root union-find W.dsu: hook the larger root under the smaller
// one, then shortcut every member to its root, until a round changes
// nothing (compute_orbits_fast's DSU, perm_group.cpp:60-116).  pm must map
// the member set onto itself.  False if the rounds do not converge.
template <bool kCg>
__device__ __forceinline__ bool sp_dsu_apply(const uint16_t* pm, const uint32_t* members,
                                          uint32_t count, uint32_t n) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  volatile uint32_t* dsu = W.dsu;
  for (uint32_t round = 0;; ++round) {
    if (round > count + 1) return false;
    bool changed = false;
    for (uint32_t i = lane; i < count; i += 32) {
      const uint32_t v = members[i];
      const uint32_t img = ldx<kCg>(pm + v);
      if (img == v) continue;
      const uint32_t a = sp_find(dsu, v, n), b = sp_find(dsu, img, n);
      if (a != b) {
        atomicMin((uint32_t*)&dsu[max(a, b)], min(a, b));
        changed = true;
      }
    }
    __syncwarp();
    for (uint32_t i = lane; i < count; i += 32) {
      const uint32_t v = members[i];
      atomicMin((uint32_t*)&dsu[v], sp_find(dsu, v, n));
    }
    __syncwarp();
    if (!__any_sync(GCL_FULL, changed)) return true;
  }
}

// subgroup_fixing_sequence + compute_orbits_fast (perm_group.cpp:5-116).
// The reference unites v with aut[v] over all vertices; an automorphism that
// fixes the sequence maps the node's partition onto itself, cell by cell, so
// the orbits that meet the target cell lie inside it and are found by
// uniting over the cell's members alone (O(cell) per automorphism instead of
// O(n)); the least vertex of each orbit -- the representative -- is the same.
template <bool kCg = false>
__device__ __forceinline__ bool sp_orbits(int idx, int num_aut, uint32_t seqlen) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n;
  SpTc t = W.tc[idx];
  const int limit = num_aut < (int)W.max_aut ? num_aut : (int)W.max_aut;
  const int from = t.last == -1 ? 0 : t.last;
  volatile uint32_t* dsu = W.dsu;
  const uint32_t* reps = t.rslot >= 0 ? W.reps + (uint64_t)t.rslot * W.stride : nullptr;
  const uint32_t* mem = W.elem + t.first;
  for (uint32_t i = lane; i < t.len; i += 32) {
    const uint32_t v = mem[i];
    dsu[v] = reps ? reps[v] : v;
  }
  __syncwarp();
  bool any = false;
  // the store entries that fix the sequence, 32 at a time (one per lane),
  // each batch merged in one union-find pass over (entry, member) pairs
  for (int base = from; base < limit; base += 32) {
    const int a = base + (int)lane;
    bool fix = a < limit;
    if (fix) {
      // extend what is known about entry a along the current sequence: the
      // prefix it fixes and the first position it moves stay valid until a
      // backtrack shortens the sequence below them (sp_fix_clamp)
      const bool kept = (uint32_t)a < W.fixcap;
      uint2 st = kept ? W.fixst[a] : make_uint2(0u, kNone);
      if (st.y != kNone && st.y < seqlen) {
        fix = false;
      } else {
        const uint16_t* pa = W.auts + (uint64_t)a * W.stride;
        uint32_t j = st.x;
        for (; j < seqlen; ++j) {
          const uint32_t sv = W.seq[j];
          if (ldx<kCg>(pa + sv) != sv) break;
        }
        fix = j >= seqlen;
        st.x = j;
        st.y = fix ? kNone : j;
        if (kept) W.fixst[a] = st;
      }
    }
    const uint32_t fm = __ballot_sync(GCL_FULL, fix);
    if (!fm) continue;
    any = true;
    const uint32_t nf = (uint32_t)__popc(fm);
    // the cell must map onto itself (a failed check is an internal error)
    bool out = false;
    for (uint32_t x = lane; x < nf * t.len; x += 32) {
      const uint32_t which = (uint32_t)__fns(fm, 0, (int)(x / t.len) + 1);
      const uint16_t* pm = W.auts + (uint64_t)(base + (int)which) * W.stride;
      const uint32_t q = W.pos[ldx<kCg>(pm + mem[x % t.len])];
      out |= q < t.first || q >= t.first + t.len;
    }
    if (__any_sync(GCL_FULL, out)) return false;
    for (uint32_t round = 0;; ++round) {
      if (round > t.len + 1) return false;
      bool changed = false;
      for (uint32_t x = lane; x < nf * t.len; x += 32) {
        const uint32_t which = (uint32_t)__fns(fm, 0, (int)(x / t.len) + 1);
        const uint16_t* pm = W.auts + (uint64_t)(base + (int)which) * W.stride;
        const uint32_t v = mem[x % t.len];
        const uint32_t img = ldx<kCg>(pm + v);
        if (img == v) continue;
        const uint32_t ra = sp_find(dsu, v, n), rb = sp_find(dsu, img, n);
        if (ra != rb) {
          atomicMin((uint32_t*)&dsu[max(ra, rb)], min(ra, rb));
          changed = true;
        }
      }
      __syncwarp();
      for (uint32_t i = lane; i < t.len; i += 32) {
        const uint32_t v = mem[i];
        atomicMin((uint32_t*)&dsu[v], sp_find(dsu, v, n));
      }
      __syncwarp();
      if (!__any_sync(GCL_FULL, changed)) break;
    }
  }
  if (!any) return true;
  if (t.rslot < 0) {
    if (W.pool_top >= W.pool_cap) return false;  // caller reports overflow
    t.rslot = (int32_t)W.pool_top;
    __syncwarp();
    if (lane == 0) {
      W.pool_owner[W.pool_top] = idx;
      W.pool_top += 1;
      W.tc[idx].rslot = t.rslot;
    }
    __syncwarp();
  }
  uint32_t* rw = W.reps + (uint64_t)t.rslot * W.stride;
  for (uint32_t i = lane; i < t.len; i += 32) {
    const uint32_t v = mem[i];
    rw[v] = sp_find(dsu, v, n);
  }
  __syncwarp();
  return true;
}

// After a backtrack to sequence length s: positions >= s of the sequence
// change, so what entries [0, count) knew about them is dropped.
__device__ __forceinline__ void sp_fix_clamp(uint32_t s, uint32_t count) {
  SpWarp& W = sp_w();
  count = min(count, W.fixcap);
  for (uint32_t a = lane_id(); a < count; a += 32) {
    uint2 st = W.fixst[a];
    if (st.x > s || (st.y != kNone && st.y >= s)) {
      st.x = min(st.x, s);
      if (st.y != kNone && st.y >= s) st.y = kNone;
      W.fixst[a] = st;
    }
  }
  __syncwarp();
}

// aut[label[j]] = elem[j] (sequential.cpp:505-520, 544-555)
__device__ __forceinline__ void sp_store_aut(const uint32_t* label, uint16_t* dst) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  for (uint32_t j = lane; j < W.n; j += 32) dst[label[j]] = (uint16_t)W.elem[j];
  __syncwarp();
}

// Colour partition (initializePartition_s, partition_refinement.cpp:28-68):
// a stable LSD radix sort of the identity order by colour.
__device__ __noinline__ void sp_init_partition(const int32_t* color) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n;
  for (uint32_t i = lane; i < n; i += 32) W.elem[i] = i;
  __syncwarp();
  bool colored = false;
  if (color)
    for (uint32_t i = lane; i < n; i += 32) colored |= color[i] != 0;
  colored = __any_sync(GCL_FULL, colored);
  if (colored) {
    uint32_t* a = W.elem;
    uint32_t* b = W.tmp;
    for (int pass = 0; pass < 4; ++pass) {
      const int sh = pass * 8;
      for (uint32_t i = lane; i < 256; i += 32) W.hist[i] = 0;
      __syncwarp();
      for (uint32_t i = lane; i < n; i += 32) {
        const uint32_t key = (uint32_t)color[a[i]] ^ 0x80000000u;
        atomicAdd(&W.hist[(key >> sh) & 255u], 1u);
      }
      __syncwarp();
      if (lane == 0) {
        uint32_t run = 0;
        for (int d = 0; d < 256; ++d) {
          W.pre[d] = run;
          run += W.hist[d];
        }
      }
      __syncwarp();
      // stable scatter: one lane walks the digits in order
      if (lane == 0)
        for (uint32_t i = 0; i < n; ++i) {
          const uint32_t key = (uint32_t)color[a[i]] ^ 0x80000000u;
          b[W.pre[(key >> sh) & 255u]++] = a[i];
        }
      __syncwarp();
      uint32_t* t = a;
      a = b;
      b = t;
    }
    // four passes: the result is back in elem
  }
  for (uint32_t i = lane; i < n; i += 32) W.pos[W.elem[i]] = i;
  for (uint32_t w = lane; w < W.nw; w += 32) {
    W.stb[w] = 0;
    W.act[w] = 0;
    W.tcb[w] = 0;
  }
  for (uint32_t i = lane; i < n; i += 32) {
    W.cnt[i] = 0;
    W.cellcnt[i] = 0;
    W.fill[i] = 0;
    W.inlev[i] = 0;
  }
  __syncwarp();
  // cell starts where the colour changes
  for (uint32_t i = lane; i < n; i += 32) {
    const bool st = i == 0 || (color && color[W.elem[i]] != color[W.elem[i - 1]]);
    if (st) atomicOr((unsigned long long*)&W.stb[i >> 6], (unsigned long long)bit64(i & 63));
  }
  __syncwarp();
  bm_resummarize(W.stb, W.sts, W.nw, W.nsw);
  uint32_t cells = 0;
  for (uint32_t w = lane; w < W.nw; w += 32) cells += popc64(W.stb[w]);
  cells = __reduce_add_sync(GCL_FULL, cells);
  // every cell starts active (sequential.cpp:628, refinement with no subsequence)
  for (uint32_t w = lane; w < W.nw; w += 32) W.act[w] = W.stb[w];
  __syncwarp();
  bm_resummarize(W.act, W.acts, W.nw, W.nsw);
  for (uint32_t w = lane; w < W.nsw; w += 32) W.tcbs[w] = 0;
  if (lane == 0) {
    W.ncells = cells;
    W.nact = cells;
  }
  __syncwarp();
}

// Input checks: indices in range, rows strictly ascending (so no duplicate
// edge), no loop, and both directions of every edge stored.
__device__ __noinline__ bool sp_check_input(int64_t m) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n;
  bool bad = W.rp[0] != 0 || (int64_t)W.rp[n] != m;
  for (uint32_t v = lane; v < n && !bad; v += 32) {
    const int32_t b = W.rp[v], e = W.rp[v + 1];
    if (b < 0 || e < b || (int64_t)e > m) {
      bad = true;
      break;
    }
    int32_t prev = -1;
    for (int32_t i = b; i < e; ++i) {
      const int32_t u = W.col[i];
      if (u <= prev || (uint32_t)u >= n || (uint32_t)u == v) {
        bad = true;
        break;
      }
      prev = u;
    }
  }
  if (__any_sync(GCL_FULL, bad)) return false;
  for (uint32_t v = lane; v < n && !bad; v += 32) {
    const int32_t b = W.rp[v], e = W.rp[v + 1];
    for (int32_t i = b; i < e && !bad; ++i) {
      const uint32_t u = (uint32_t)W.col[i];
      int32_t lo = W.rp[u], hi = W.rp[u + 1] - 1;
      bool found = false;
      while (lo <= hi) {
        const int32_t mid = (lo + hi) >> 1;
        const uint32_t x = (uint32_t)W.col[mid];
        if (x == v) {
          found = true;
          break;
        }
        if (x < v)
          lo = mid + 1;
        else
          hi = mid - 1;
      }
      if (!found) bad = true;
    }
  }
  return !__any_sync(GCL_FULL, bad);
}

struct SpArgs {
  BatchArgs A;
  const int* list;   // graph ids to process
  const int* count;  // number of ids (device)
  int* next;         // work counter
  int* fail_list;    // graphs needing the rerun pass
  int* fail_count;
  uint32_t n_max;
  uint64_t m2_max;
  uint32_t pool;
  uint32_t cap;
  uint64_t slot_bytes;
};

struct SpResult {
  int32_t status;
  int num_aut;
  int64_t nodes;
};

// Point the warp's arrays into its slot (and its shared-memory region when
// the per-step arrays fit there).  Lane 0 writes; the caller syncs the warp.
__device__ __noinline__ void sp_bind(uint8_t* slot, const SpLayout& Lo, uint32_t n,
                                     const int32_t* rp, const int32_t* col, uint8_t* smem,
                                     uint64_t smem_bytes, uint32_t pool, uint32_t cap,
                                     uint32_t max_aut) {
  SpWarp& W = sp_w();
  if (lane_id() != 0) return;
  // the n-sized u32 arrays
  uint32_t* base[26];
  for (int i = 0; i < 26; ++i) base[i] = (uint32_t*)(slot + Lo.u32n[i]);
  W.elem = base[0];
  W.pos = base[1];
  W.inlev = base[2];
  W.cnt = base[3];
  W.T = base[4];
  W.Tc = base[5];
  W.cellcnt = base[6];
  W.off = base[7];
  W.fill = base[8];
  W.G = base[9];
  W.tmp = base[10];
  W.lst1 = base[11];
  W.lst2 = base[12];
  W.seq = base[13];
  W.fseq = base[14];
  W.bseq = base[15];
  W.flabel = base[16];
  W.blabel = base[17];
  W.dsu = base[18];
  W.hist = base[19];
  W.pre = base[20];
  W.fpos = base[21];
  W.bpos = base[22];
  W.nsl = base[23];
  W.pathcode = (int32_t*)base[24];
  W.umark = base[25];
  W.ulog = (uint2*)(slot + Lo.ulog);
  W.fixst = (uint2*)(slot + Lo.fixst);
  W.fixcap = Lo.fixcap;
  W.ulog_cap = Lo.ulog_cap;
  W.utop = 0;
  W.ulog_bad = 0;
  W.fcode = (int32_t*)(slot + Lo.fcode);
  W.ccode = (int32_t*)(slot + Lo.ccode);
  W.pool_owner = (int32_t*)(slot + Lo.pool_owner);
  W.stb = (uint64_t*)(slot + Lo.stb);
  W.sts = (uint64_t*)(slot + Lo.sts);
  W.act = (uint64_t*)(slot + Lo.act);
  W.acts = (uint64_t*)(slot + Lo.acts);
  W.tcb = (uint64_t*)(slot + Lo.tcb);
  W.tcbs = (uint64_t*)(slot + Lo.tcbs);
  W.fcert = (uint32_t*)(slot + Lo.fcert);
  W.bcert = (uint32_t*)(slot + Lo.bcert);
  W.ccert = (uint32_t*)(slot + Lo.ccert);
  W.tc = (SpTc*)(slot + Lo.tc);
  W.reps = (uint32_t*)(slot + Lo.reps);
  W.auts = (uint16_t*)(slot + Lo.auts);
  W.rp = rp;
  W.col = col;
  W.n = n;
  W.nw = (n + 63) / 64 + 1;
  W.nsw = (W.nw + 63) / 64 + 1;
  W.stride = Lo.stride;
  W.npend = 0;
  if (smem && sp_smem_bytes(n) <= smem_bytes) {
    // stage the per-step arrays in this warp's shared memory
    const uint64_t a = (((uint64_t)n + 2) * 4u + 15) & ~15ull;
    const uint32_t nw2 = W.nw, nsw2 = W.nsw;
    uint8_t* q = smem;
    W.elem = (uint32_t*)q;
    q += a;
    W.pos = (uint32_t*)q;
    q += a;
    W.inlev = (uint32_t*)q;
    q += a;
    W.nsl = (uint32_t*)q;
    q += a;
    W.stb = (uint64_t*)q;
    q += 8 * nw2;
    W.sts = (uint64_t*)q;
    q += 8 * nsw2;
    W.act = (uint64_t*)q;
    q += 8 * nw2;
    W.acts = (uint64_t*)q;
    q += 8 * nsw2;
    W.tcb = (uint64_t*)q;
    q += 8 * nw2;
    W.tcbs = (uint64_t*)q;
  }
  W.pool_top = 0;
  W.pool_cap = pool;
  W.aut_cap = cap;
  W.max_aut = max_aut;
  W.ntouched = 0;
}

__device__ __noinline__ SpResult sp_search(const BatchArgs& A, int g, uint8_t* slot,
                                           const SpLayout& Lo, uint32_t pool, uint32_t cap,
                                           uint8_t* smem, uint64_t smem_bytes) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const int64_t vo = A.voff[g];
  const uint32_t n = (uint32_t)(A.voff[g + 1] - vo);
  const int64_t eo = A.eoff[g];
  const int64_t m = A.eoff[g + 1] - eo;
  SpResult res{kOk, 0, 1};
  if (n == 0) return res;
  sp_bind(slot, Lo, n, A.rowptr + vo + g, A.col + eo, smem, smem_bytes, pool, cap, A.max_aut);
  __syncwarp();
  if (!sp_check_input(m)) {
    res.status = kBadInput;
    return res;
  }
  uint64_t deadline = 0;
  if (A.budget_ns)
    deadline = __shfl_sync(GCL_FULL, lane == 0 ? global_ns() : 0ull, 0) + A.budget_ns;
  sp_init_partition(A.color ? A.color + vo : nullptr);

  uint32_t level = 0, seqlen = 0, eqlevfirst = 0, first_seqlen = 0, best_seqlen = 0;
  int code = 0, canon_level = 0, eqlevcanon = 0, comp_canon = 0, tcl = 0, num_aut = 0;
  bool first_found = false;
  int64_t nodes = 1;
  int32_t status = kOk;
  bool pending = true;  // root refinement with every cell active
  uint64_t iter = 0;
  while (true) {
    if (pending) {
      pending = false;
      code = sp_refine(level);
      if (code < 0) {
        status = kInternal;
        break;
      }
      ++level;
      __syncwarp();
      if (lane == 0) {
        W.fcode[level - 1] = code;
        if (level == 1) W.utop = 0;  // the root partition is never undone
      }
      __syncwarp();
      continue;
    }
    if (level == 0) break;
    if ((++iter & 15) == 0 && deadline &&
        __shfl_sync(GCL_FULL, lane == 0 ? global_ns() : 0ull, 0) > deadline) {
      status = kTimeout;
      break;
    }
    int bt = -1, descend = -1;
    bool classify = false;
    const bool disc = W.ncells == n;
    if (!first_found) {
      if (disc) {
        // first_terminal (sequential.cpp:259-303)
        sp_leaf_cert(W.fcert);
        sp_copy_u32(W.bcert, W.fcert, (uint32_t)m);
        sp_copy_u32(W.flabel, W.elem, n);
        sp_copy_u32(W.blabel, W.elem, n);
        sp_copy_u32(W.fseq, W.seq, seqlen);
        sp_copy_u32(W.bseq, W.seq, seqlen);
        sp_copy_u32((uint32_t*)W.ccode, (const uint32_t*)W.fcode, level);
        if (lane == 0) {
          W.fcode[level] = kSentinel;
          W.ccode[level] = kSentinel;
        }
        __syncwarp();
        eqlevfirst = level;
        first_seqlen = best_seqlen = seqlen;
        first_found = true;
        canon_level = eqlevcanon = (int)level;
        comp_canon = 0;
        bt = (int)level - 1;
      } else {
        const uint32_t t = sp_first_nonsingleton();
        if (t == kNone || tcl > (int)n) {
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
        descend = tcl - 1;
      }
    } else {
      classify = true;
      if (!disc && (eqlevfirst == level || comp_canon >= 0)) {
        if (tcl < (int)level) {
          const uint32_t t = sp_first_nonsingleton();
          if (t == kNone || tcl > (int)n) {
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
          classify = false;
        } else {
          if (num_aut > 0 && num_aut > W.tc[idx].last) {
            if (!sp_orbits(idx, num_aut, seqlen)) {
              status = W.pool_top >= W.pool_cap ? kAutOverflow : kInternal;
              break;
            }
            __syncwarp();
            if (lane == 0) W.tc[idx].last = num_aut;
            __syncwarp();
          }
          descend = idx;
        }
      }
    }
    if (descend >= 0) {
      const SpTc t = W.tc[descend];
      const uint32_t v = sp_next_rep(t);
      if (v == kNone) {
        __syncwarp();
        if (lane == 0) W.tc[descend].counter = n;
        __syncwarp();
        bt = (int)level - 1;
        classify = false;
      } else {
        __syncwarp();
        if (lane == 0) {
          W.tc[descend].counter = v + 1;
          W.seq[seqlen] = v;
        }
        __syncwarp();
        ++seqlen;
        ++nodes;
        if (sp_individualize(level, v, t.first)) {
          if (!first_found) {
            pending = true;
            continue;
          }
          code = sp_refine(level);
          if (code < 0) {
            status = kInternal;
            break;
          }
          ++level;
        } else if (!first_found) {
          __syncwarp();
          if (lane == 0) W.fcode[level - 1] = code;
          __syncwarp();
          continue;
        }
      }
    }
    if (classify) {
      // classify_node (sequential.cpp:396-624)
      const uint32_t Lv = level;
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
        sp_leaf_cert(W.ccert);
        if (eqlevfirst == Lv && sp_cmp_leaf(W.ccert, W.flabel, W.fcert, false) == 0) dec = 1;
        if (dec == 0) {
          if (comp_canon == 0) {
            if ((int)Lv < canon_level)
              comp_canon = 1;
            else
              comp_canon = sp_cmp_leaf(W.ccert, W.blabel, W.bcert, true);
          }
          dec = comp_canon == 0 ? 2 : (comp_canon > 0 ? 3 : 4);
        }
      }
      if (dec == 1 || dec == 2) {
        const uint32_t si = (uint32_t)num_aut % W.max_aut;
        if (si >= W.aut_cap) {
          status = kAutOverflow;
          break;
        }
        sp_store_aut(dec == 1 ? W.flabel : W.blabel, W.auts + (uint64_t)si * W.stride);
        if (lane == 0 && si < W.fixcap) W.fixst[si] = make_uint2(0u, kNone);
        __syncwarp();
        ++num_aut;
        const int gg = dec == 1 ? sp_gca(W.fseq, first_seqlen, seqlen)
                                : sp_gca(W.bseq, best_seqlen, seqlen);
        bt = gg >= 0 ? gg : (int)Lv - 1;
      } else if (dec == 3) {
        canon_level = eqlevcanon = (int)Lv;
        comp_canon = 0;
        sp_copy_u32(W.bcert, W.ccert, (uint32_t)m);
        sp_copy_u32(W.blabel, W.elem, n);
        sp_copy_u32(W.bseq, W.seq, seqlen);
        if (lane == 0) W.ccode[Lv] = kSentinel;
        __syncwarp();
        best_seqlen = seqlen;
        bt = (int)Lv - 1;
      } else if (dec == 4) {
        bt = (int)Lv - 1;
      }
    }
    if (bt >= 0) {
      // backtrack_to (sequential.cpp:650-670)
      const uint32_t Lv = (uint32_t)bt;
      if (Lv == 0) {
        level = 0;
        continue;
      }
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
      sp_fix_clamp(seqlen, (uint32_t)min(num_aut, (int)W.max_aut));
      // representative arrays of levels deeper than Lv are free again
      __syncwarp();
      if (lane == 0)
        while (W.pool_top > 0 && W.pool_owner[W.pool_top - 1] >= (int32_t)Lv) W.pool_top -= 1;
      __syncwarp();
    }
  }
  res.status = status;
  res.num_aut = num_aut;
  res.nodes = nodes;
  return res;
}

// Outputs from the best leaf: labeling and the dense canonical matrix.
__device__ __noinline__ void sp_write_outputs(const BatchArgs& A, int g) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n;
  const int64_t vo = A.voff[g];
  if (A.out_label)
    for (uint32_t j = lane; j < n; j += 32) A.out_label[vo + j] = (int32_t)W.blabel[j];
  if (A.out_rows) {  // row i: bit j set iff canonical i ~ j, ceil(n/64) words
    const uint32_t words = (n + 63) / 64;
    uint64_t* o = A.out_rows + A.roff[g];
    for (uint32_t i = lane; i < n; i += 32) {
      uint64_t* row = o + (uint64_t)i * words;
      for (uint32_t w = 0; w < words; ++w) row[w] = 0;
      const uint32_t v = W.blabel[i];
      for (int32_t j = W.rp[v]; j < W.rp[v + 1]; ++j) {
        const uint32_t c = W.bcert[j];
        row[c >> 6] |= bit64(c & 63);
      }
    }
  }
  if (A.out_dense) {
    uint8_t* o = A.out_dense + A.ooff[g];
    const uint64_t nn = (uint64_t)n * n;
    for (uint64_t i = lane; i < nn; i += 32) o[i] = 0;
    __syncwarp();
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t v = W.blabel[i];
      const int32_t b = W.rp[v], e = W.rp[v + 1];
      for (int32_t j = b + (int32_t)lane; j < e; j += 32) o[(uint64_t)i * n + W.bcert[j]] = 1;
    }
  }
  __syncwarp();
}

}  // namespace gcl
