// canon_warp64.cuh -- one warp canonizes one graph with n <= 64 vertices.
//
// The search is the reference's sequential individualization-refinement DFS
// (src/sequential.cpp:216-670) step for step, so the canonical form, the
// number of stored automorphisms and the number of search-tree nodes equal
// the reference's on every input.  What changes is the representation:
//
//   * a vertex set is one 64-bit mask; lane L owns vertices L and L+32;
//   * the ordered partition is vertex-indexed: each vertex knows the start
//     position `cs` of its cell and the member mask `cm` of that cell, and the
//     warp holds `starts`, the mask of cell start positions.  The order of
//     vertices inside a cell is never stored: the reference's refinement and
//     search depend only on the cells as sets (fragments are ordered by count,
//     targets and branch vertices are chosen by position and by vertex id),
//     so leaves, codes and pruning decisions are unchanged;
//   * counting neighbours in a splitter is popc(adj[v] & splitter); splitting
//     every cell at once is a radix pass over the count bits with warp
//     ballots; only the invariant hash (a serial chain, order-dependent) is
//     folded by lane 0 over the split cells in position order;
//   * a leaf certificate is one 64-bit row per canonical vertex; the
//     reference's n^2 upper-triangle compare (sequential.cpp:114-124) becomes
//     a masked row compare plus a warp min, and the isAutomorphism test
//     against the first leaf (sequential.cpp:127-167) becomes certificate
//     equality, which is the same predicate for a bijection.
#pragma once
#include <cstdint>

#include "gcl_device.cuh"

namespace gcl {

constexpr int kW64MaxN = 64;
constexpr int kW64Levels = kW64MaxN + 2;

enum GraphStatus : int32_t {
  kOk = 0,
  kAutOverflow = 1,  // automorphism store too small for this graph: rerun
  kTooLarge = 2,     // n above this kernel's limit
  kBadInput = 3,     // loop, duplicate or one-directional edge, bad index
  kInternal = 4,     // an internal consistency check failed (no result)
  kTimeout = 5,      // the per-graph time budget ran out (no result)
};

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Target cell of one search level (TargetCell, structs.h:10-17).  `members`
// replaces elems[v] != -1, `repmask` the test elems[v] == v; the orbit
// representatives themselves live in the slot workspace and are only valid
// once an orbit computation has run (`reps_valid`).
struct TcHdr {
  uint64_t members;
  uint64_t repmask;
  int32_t last;  // last_num_aut_at_level
  uint16_t counter;
  uint8_t first;
  uint8_t reps_valid;
};

struct __align__(16) W64Smem {
  uint64_t adj[kW64MaxN];
  uint64_t first_cert[kW64MaxN];  // first leaf, row per canonical vertex
  uint64_t best_cert[kW64MaxN];   // best leaf
  TcHdr tc[kW64Levels];
  uint32_t dsu[kW64MaxN];
  uint16_t firstcode[kW64Levels];
  uint16_t canoncode[kW64Levels];
  uint8_t inlev[kW64MaxN];  // in_level of the cell starting at a position
  uint8_t fk[kW64MaxN];     // count value of the fragment starting at a position
  uint8_t seq[kW64MaxN];
  uint8_t first_seq[kW64MaxN];
  uint8_t best_seq[kW64MaxN];
  uint8_t map[kW64MaxN];
};

struct BatchArgs {
  int count;
  const int64_t* voff;   // [count+1]
  const int64_t* eoff;   // [count+1]
  const int32_t* rowptr; // arena, graph g at voff[g] + g
  const int32_t* col;    // arena, graph g at eoff[g]
  const int32_t* color;  // arena at voff[g], or null
  const int32_t* order;  // processing order of graph ids, or null
  uint32_t max_aut;
  uint32_t aut_cap;      // automorphism slots per workspace slot (<= max_aut)
  uint8_t* out_dense;    // n*n bytes per graph at ooff[g], or null
  const int64_t* ooff;
  uint64_t* out_cert;    // n rows per graph at voff[g], or null
  int32_t* out_label;    // n per graph at voff[g], or null
  int64_t* out_stats;    // {num_aut, nodes} per graph, or null
  int32_t* status;       // per graph
  uint8_t* work;         // per-warp slot workspace
  uint64_t slot_bytes;
  uint64_t budget_ns;    // per-graph time budget (0 = unlimited)
};

// Per-slot workspace layout: reps[kW64Levels][64] then the automorphism ring.
__host__ __device__ constexpr uint64_t w64_slot_bytes(uint32_t aut_cap) {
  return ((uint64_t)kW64Levels * 64u + (uint64_t)aut_cap * 64u + 255u) & ~255ull;
}

template <int VPL>
struct W64Lane {
  uint64_t adj[VPL];
  uint64_t cm[VPL];
  uint32_t cs[VPL];
  uint32_t fpos[VPL];
  uint32_t bpos[VPL];
};

template <int VPL>
__device__ __forceinline__ uint64_t ballot64(const bool (&b)[VPL]) {
  uint64_t m = __ballot_sync(GCL_FULL, b[0]);
  if (VPL > 1) m |= (uint64_t)__ballot_sync(GCL_FULL, b[VPL > 1 ? 1 : 0]) << 32;
  return m;
}

template <int VPL>
class W64Search {
 public:
  __device__ W64Search(W64Smem& s, const BatchArgs& a, int n, uint8_t* slot)
      : S(s), A(a), n(n), reps(slot), auts(slot + (uint64_t)kW64Levels * 64u) {
    lane = lane_id();
    full = low_mask((uint32_t)n);
  }

  W64Smem& S;
  const BatchArgs& A;
  const int n;
  uint8_t* reps;
  uint8_t* auts;
  uint32_t lane;
  uint64_t full;
  W64Lane<VPL> L;

  // search state (warp-uniform), Nauty_Sequential members (sequential.h:24-45)
  uint64_t starts = 0;
  uint32_t level = 0, seqlen = 0;
  int code = 0;
  int canon_level = 0, eqlevcanon = 0, comp_canon = 0;
  uint32_t eqlevfirst = 0;
  int tcl = 0;
  bool first_found = false;
  uint32_t first_seqlen = 0, best_seqlen = 0;
  int num_aut = 0;
  int64_t nodes = 0;
  int32_t status = kOk;
  uint64_t deadline = 0;

  // Records a failure (warp-uniform); every caller that indexes by level
  // checks `status` afterwards and the search loop stops.
  __device__ __forceinline__ void fail(int32_t st) {
    if (status == kOk) status = st;
  }
  __device__ __forceinline__ bool out_of_time() {
    if (!deadline) return false;
    const uint64_t t = __shfl_sync(GCL_FULL, lane == 0 ? global_ns() : 0ull, 0);
    return t > deadline;
  }

  __device__ __forceinline__ uint32_t vid(int k) const { return lane + 32u * (uint32_t)k; }
  __device__ __forceinline__ bool valid(int k) const { return vid(k) < (uint32_t)n; }

  // ---- set-up: adjacency masks and the colour partition -------------------
  __device__ bool load(int64_t vo, const int32_t* rp, const int32_t* cl, const int32_t* color,
                       int64_t m) {
    bool bad = false;
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      uint64_t a = 0;
      if (valid(k)) {
        const uint32_t v = vid(k);
        const int32_t b = rp[v], e = rp[v + 1];
        if (b < 0 || e < b || (int64_t)e > m) bad = true;
        for (int32_t i = b; i < e && !bad; ++i) {
          const int32_t u = cl[i];
          if (u < 0 || u >= n || (uint32_t)u == v || ((a >> u) & 1ull)) { bad = true; break; }
          a |= 1ull << u;
        }
        S.adj[v] = a;
      }
      L.adj[k] = a;
    }
    __syncwarp();
    // symmetric adjacency (CSRGraph::fromDIMACS inserts both directions)
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      uint64_t a = L.adj[k];
      while (a && !bad) {
        const uint32_t u = ctz64(a);
        a &= a - 1;
        if (!((S.adj[u] >> vid(k)) & 1ull)) bad = true;
      }
    }
    if (__any_sync(GCL_FULL, bad)) return false;

    // initializePartition_s (partition_refinement.cpp:28-68): cells are the
    // colour classes in ascending colour order.
    int32_t c[VPL];
    bool colored = false;
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      c[k] = (color && valid(k)) ? color[vo + vid(k)] : 0;
      colored |= c[k] != 0;
    }
    if (!__any_sync(GCL_FULL, colored)) {
#pragma unroll
      for (int k = 0; k < VPL; ++k) {
        L.cs[k] = 0;
        L.cm[k] = full;
      }
      starts = n > 0 ? 1ull : 0ull;
    } else {
      int32_t* ctmp = reinterpret_cast<int32_t*>(S.dsu);
#pragma unroll
      for (int k = 0; k < VPL; ++k)
        if (valid(k)) ctmp[vid(k)] = c[k];
      __syncwarp();
      uint64_t st = 0;
#pragma unroll
      for (int k = 0; k < VPL; ++k) {
        uint32_t below = 0;
        uint64_t same = 0;
        if (valid(k))
          for (int u = 0; u < n; ++u) {
            const int32_t cu = ctmp[u];
            below += cu < c[k];
            same |= (uint64_t)(cu == c[k]) << u;
          }
        L.cs[k] = below;
        L.cm[k] = same;
        if (valid(k)) st |= 1ull << below;
      }
      starts = warp_or64(st);
      __syncwarp();
    }
#pragma unroll
    for (int k = 0; k < VPL; ++k)
      if (valid(k)) S.inlev[vid(k)] = 0;
    __syncwarp();
    return true;
  }

  // ---- Partition_s_refinement (partition_refinement.cpp:150-485) -----------
  __device__ int refine(uint64_t active) {
    uint32_t lc = popc64(starts);
    uint32_t hint = 0;
    uint32_t iters = 0;
    while (starts != full && active) {
      if (++iters > 64u * 64u + 64u) {  // each step removes an active cell or splits one
        fail(kInternal);
        return 0;
      }
      uint32_t s;
      if ((active >> hint) & 1ull) {
        s = hint;
      } else {
        const uint64_t a = active & ge_mask(hint + 1);
        s = ctz64(a ? a : active);
      }
      active &= ~(1ull << s);
      const uint64_t nx = starts & ge_mask(s + 1);
      const uint32_t e = nx ? ctz64(nx) : (uint32_t)n;
      const uint32_t len = e - s;
      lc = mash(lc, s + e - 1);  // split1 + split2
      if (len > 1) lc = mash(lc, len);

      bool insp[VPL];
#pragma unroll
      for (int k = 0; k < VPL; ++k) insp[k] = valid(k) && L.cs[k] == s;
      const uint64_t spl = ballot64<VPL>(insp);  // splitter members

      if (len == 1) {
        // singleton splitter: every cell meeting N(w) partially splits into
        // [neighbours, non-neighbours]
        if (popc64(spl) != 1) {
          fail(kInternal);
          return 0;
        }
        const uint64_t N = S.adj[ctz64(spl)];
        uint64_t ns = 0;
#pragma unroll
        for (int k = 0; k < VPL; ++k) {
          if (!valid(k)) continue;
          const uint64_t C = L.cm[k], CN = C & N;
          if (CN != 0 && CN != C) {
            if ((N >> vid(k)) & 1ull) {
              L.cm[k] = CN;
            } else {
              L.cm[k] = C & ~N;
              L.cs[k] += popc64(CN);
              ns |= 1ull << L.cs[k];
            }
          }
        }
        const uint64_t NS = warp_or64(ns);
        if (NS) {
          uint32_t o_lc = lc, o_hint = hint;
          uint64_t o_act = active;
          if (lane == 0) {
            const uint64_t all = starts | NS;
            uint64_t t = NS;
            while (t) {
              const uint32_t p = ctz64(t);
              t &= t - 1;
              const uint32_t c = msb64(starts & low_mask(p));
              const uint64_t q = all & ge_mask(p + 1);
              const uint32_t qe = q ? ctz64(q) : (uint32_t)n;
              const uint32_t nb = p - c, nn = qe - p;
              o_lc = mash(o_lc, p - 1);  // cell.first + neighbors_size - 1
              const uint8_t old = S.inlev[c];
              S.inlev[c] = (uint8_t)(level + 1);
              S.inlev[p] = old;
              if (((o_act >> c) & 1ull) || nb >= nn) {
                o_act |= 1ull << p;
                if (nn == 1) o_hint = p;
              } else {
                o_act |= 1ull << c;
                if (nb == 1) o_hint = c;
              }
            }
          }
          __syncwarp();
          lc = __shfl_sync(GCL_FULL, o_lc, 0);
          hint = __shfl_sync(GCL_FULL, o_hint, 0);
          active = bcast64(o_act, 0);
          starts |= NS;
        }
      } else {
        // non-singleton splitter: split by neighbour count, fragments in
        // ascending count order
        uint32_t cnt[VPL];
        uint32_t mx = 0;
#pragma unroll
        for (int k = 0; k < VPL; ++k) {
          cnt[k] = valid(k) ? popc64(L.adj[k] & spl) : 0u;
          mx = max(mx, cnt[k]);
        }
        mx = __reduce_max_sync(GCL_FULL, mx);
        uint64_t eq[VPL];
        uint32_t lt[VPL];
#pragma unroll
        for (int k = 0; k < VPL; ++k) {
          eq[k] = L.cm[k];
          lt[k] = 0;
        }
        for (int b = mx ? 31 - __clz(mx) : -1; b >= 0; --b) {
          bool bit[VPL];
#pragma unroll
          for (int k = 0; k < VPL; ++k) bit[k] = (cnt[k] >> b) & 1u;
          const uint64_t M = ballot64<VPL>(bit);
#pragma unroll
          for (int k = 0; k < VPL; ++k) {
            if (bit[k]) {
              lt[k] += popc64(eq[k] & ~M);
              eq[k] &= M;
            } else {
              eq[k] &= ~M;
            }
          }
        }
        uint64_t ns = 0;
#pragma unroll
        for (int k = 0; k < VPL; ++k) {
          if (!valid(k)) continue;
          L.cs[k] += lt[k];
          L.cm[k] = eq[k];
          ns |= 1ull << L.cs[k];
          S.fk[L.cs[k]] = (uint8_t)cnt[k];
        }
        const uint64_t NS = warp_or64(ns) & ~starts;
        __syncwarp();
        uint32_t o_lc = lc, o_hint = hint;
        uint64_t o_act = active;
        if (lane == 0) {
          const uint64_t singles = starts & ((starts >> 1) | (1ull << (n - 1)));
          uint64_t t = starts & ~singles;
          const uint64_t all = starts | NS;
          const uint32_t lvl1 = level + 1;
          while (t) {
            const uint32_t c = ctz64(t);
            t &= t - 1;
            const uint64_t nx2 = starts & ge_mask(c + 1);
            const uint32_t end = nx2 ? ctz64(nx2) : (uint32_t)n;
            uint64_t fr = all & ge_mask(c) & low_mask(end);
            if (fr == (1ull << c)) {
              o_lc = mash(o_lc, (uint32_t)S.fk[c] + c);  // common count
              continue;
            }
            const bool was = (o_act >> c) & 1ull;
            const uint8_t old = S.inlev[c];
            uint32_t maxsz = 0, maxp = c, lastp = c;
            while (fr) {
              const uint32_t p = ctz64(fr);
              fr &= fr - 1;
              const uint32_t pe = fr ? ctz64(fr) : end;
              const uint32_t sz = pe - p;
              o_lc = mash(o_lc, (uint32_t)S.fk[p] + p);
              S.inlev[p] = (uint8_t)lvl1;
              if (sz > maxsz) {
                maxsz = sz;
                maxp = p;
              }
              if (p != c) {
                o_act |= 1ull << p;
                if (sz == 1) o_hint = p;
              }
              lastp = p;
            }
            if (!was) {
              o_act |= 1ull << c;
              o_act &= ~(1ull << maxp);
            }
            S.inlev[lastp] = old;
          }
        }
        __syncwarp();
        lc = __shfl_sync(GCL_FULL, o_lc, 0);
        hint = __shfl_sync(GCL_FULL, o_hint, 0);
        active = bcast64(o_act, 0);
        starts |= NS;
      }
    }
    lc = mash(lc, popc64(starts));
    ++level;
    return cleanup(lc);
  }

  // ---- split_by_and_refine (partition_refinement.cpp:486-539) -------------
  __device__ void individualize(uint32_t v, uint32_t t) {
    bool in[VPL];
#pragma unroll
    for (int k = 0; k < VPL; ++k) in[k] = valid(k) && L.cs[k] == t;
    const uint64_t mem = ballot64<VPL>(in);
    if (popc64(mem) == 1) return;  // singleton: nothing to split, code kept
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      if (!in[k]) continue;
      if (vid(k) == v) {
        L.cm[k] = 1ull << v;
      } else {
        L.cm[k] = mem & ~(1ull << v);
        L.cs[k] = t + 1;
      }
    }
    starts |= 1ull << (t + 1);
    if (lane == 0) {
      S.inlev[t + 1] = S.inlev[t];
      S.inlev[t] = (uint8_t)(level + 1);
    }
    __syncwarp();
    code = refine(1ull << t);
  }

  // ---- reconstruct_at_level + backtrack_to (partition_refinement.cpp:541-604,
  //      sequential.cpp:650-670) -----------------------------------------
  __device__ void backtrack(uint32_t Lv) {
    if (Lv == 0) {
      level = 0;
      return;
    }
    bool big[VPL];
    uint32_t lv[VPL];
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      const uint32_t p = vid(k);
      const bool st = valid(k) && ((starts >> p) & 1ull);
      lv[k] = st ? S.inlev[p] : 0u;
      big[k] = st && lv[k] > Lv;
    }
    const uint64_t BIG = ballot64<VPL>(big);
    if (BIG) {
      bool surv[VPL];
      uint32_t nlv[VPL];
#pragma unroll
      for (int k = 0; k < VPL; ++k) {
        const uint32_t p = vid(k);
        const bool st = valid(k) && ((starts >> p) & 1ull);
        bool sv = st;
        if (st && p > 0) {
          const uint64_t prev = starts & low_mask(p);
          if (prev && ((BIG >> msb64(prev)) & 1ull)) sv = false;
        }
        surv[k] = sv;
        nlv[k] = lv[k];
        if (sv && big[k]) {
          // the run is closed by the first following cell created at or
          // before level Lv; the merged cell takes that cell's in_level
          const uint64_t j = starts & ~BIG & ge_mask(p + 1);
          nlv[k] = j ? S.inlev[ctz64(j)] : 0xffu;
        }
      }
      const uint64_t NST = ballot64<VPL>(surv);
      bool broken[VPL];
#pragma unroll
      for (int k = 0; k < VPL; ++k) broken[k] = nlv[k] == 0xffu;
      if (ballot64<VPL>(broken)) {  // a run of new cells reached the last cell
        fail(kInternal);
        return;
      }
      __syncwarp();
#pragma unroll
      for (int k = 0; k < VPL; ++k)
        if (surv[k] && big[k]) S.inlev[vid(k)] = (uint8_t)nlv[k];
      starts = NST;
#pragma unroll
      for (int k = 0; k < VPL; ++k)
        if (valid(k)) L.cs[k] = msb64(NST & low_mask(L.cs[k] + 1));
      rebuild_cell_masks();
      __syncwarp();
    }
    if (Lv < eqlevfirst) eqlevfirst = Lv;
    if ((int)Lv <= eqlevcanon) {
      eqlevcanon = (int)Lv;
      comp_canon = 0;
    }
    seqlen = Lv - 1;
    tcl = (int)Lv;
    level = Lv;
  }

  __device__ void rebuild_cell_masks() {
    uint64_t eq[VPL];
    bool vb[VPL];
#pragma unroll
    for (int k = 0; k < VPL; ++k) vb[k] = valid(k);
    const uint64_t vm = ballot64<VPL>(vb);
#pragma unroll
    for (int k = 0; k < VPL; ++k) eq[k] = vm;
    const int nb = 32 - __clz(max(n - 1, 1));
    for (int b = nb - 1; b >= 0; --b) {
      bool bit[VPL];
#pragma unroll
      for (int k = 0; k < VPL; ++k) bit[k] = (L.cs[k] >> b) & 1u;
      const uint64_t M = ballot64<VPL>(bit);
#pragma unroll
      for (int k = 0; k < VPL; ++k) eq[k] &= bit[k] ? M : ~M;
    }
#pragma unroll
    for (int k = 0; k < VPL; ++k) L.cm[k] = valid(k) ? eq[k] : 0ull;
  }

  __device__ __forceinline__ bool discrete() const { return starts == full; }

  // target_cell_selector (partition_refinement.cpp:607-655), hint -1
  __device__ void select_tc() {
    const uint64_t singles = starts & ((starts >> 1) | (1ull << (n - 1)));
    const uint64_t ns = starts & ~singles;
    if (!ns) return;
    const uint32_t t = ctz64(ns);
    bool in[VPL];
#pragma unroll
    for (int k = 0; k < VPL; ++k) in[k] = valid(k) && L.cs[k] == t;
    const uint64_t mem = ballot64<VPL>(in);
    if (tcl >= kW64Levels) {
      fail(kInternal);
      return;
    }
    if (lane == 0) {
      TcHdr& h = S.tc[tcl];
      h.members = mem;
      h.repmask = mem;
      h.last = 0;
      h.counter = 0;
      h.first = (uint8_t)t;
      h.reps_valid = 0;
    }
    __syncwarp();
    ++tcl;
  }

  // next branch vertex: smallest v >= counter with elems[v] == v
  __device__ __forceinline__ bool next_rep(int idx) {
    const TcHdr& h = S.tc[idx];
    const uint64_t r = h.repmask & ge_mask(h.counter);
    const uint32_t c = r ? ctz64(r) : (uint32_t)n;
    __syncwarp();
    if (lane == 0) S.tc[idx].counter = (uint16_t)c;
    __syncwarp();
    return c < (uint32_t)n;
  }

  __device__ void push_and_split(int idx) {
    const uint32_t v = S.tc[idx].counter;
    const uint32_t t = S.tc[idx].first;
    __syncwarp();
    if (lane == 0) {
      S.tc[idx].counter = (uint16_t)(v + 1);
      S.seq[seqlen] = (uint8_t)v;
    }
    __syncwarp();
    ++seqlen;
    ++nodes;
    individualize(v, t);
  }

  // ---- leaves --------------------------------------------------------------
  // Certificate row of each own vertex: its neighbours renamed to positions
  // (buildPermutedFlatAdjacencyMatrixArray, CSRGraph.cpp:332-351).
  __device__ void leaf_rows(uint64_t (&R)[VPL]) {
#pragma unroll
    for (int k = 0; k < VPL; ++k)
      if (valid(k)) S.map[vid(k)] = (uint8_t)L.cs[k];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      uint64_t a = L.adj[k], r = 0;
      while (a) {
        const uint32_t u = ctz64(a);
        a &= a - 1;
        r |= 1ull << S.map[u];
      }
      R[k] = r;
    }
    __syncwarp();
  }

  // compare_adj_upper(current, stored) (sequential.cpp:114-124)
  __device__ int cmp_upper(const uint64_t (&R)[VPL], const uint64_t* B) {
    uint32_t row = 64u;
    bool sgn[VPL];
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      sgn[k] = false;
      if (!valid(k)) continue;
      const uint32_t p = L.cs[k];
      const uint64_t d = (R[k] ^ B[p]) & ge_mask(p + 1);
      if (d) {
        row = min(row, p);
        sgn[k] = (R[k] >> ctz64(d)) & 1ull;
      }
    }
    const uint32_t mrow = __reduce_min_sync(GCL_FULL, row);
    if (mrow == 64u) return 0;
    bool win[VPL];
#pragma unroll
    for (int k = 0; k < VPL; ++k) win[k] = valid(k) && L.cs[k] == mrow && sgn[k];
    return ballot64<VPL>(win) ? 1 : -1;
  }

  __device__ bool rows_equal(const uint64_t (&R)[VPL], const uint64_t* B) {
    bool ne[VPL];
#pragma unroll
    for (int k = 0; k < VPL; ++k) ne[k] = valid(k) && R[k] != B[L.cs[k]];
    return ballot64<VPL>(ne) == 0;
  }

  __device__ void store_rows(const uint64_t (&R)[VPL], uint64_t* B) {
#pragma unroll
    for (int k = 0; k < VPL; ++k)
      if (valid(k)) B[L.cs[k]] = R[k];
    __syncwarp();
  }

  __device__ void copy_seq(uint8_t* dst) {
    for (uint32_t j = lane; j < seqlen; j += 32) dst[j] = S.seq[j];
    __syncwarp();
  }

  // get_gca_level (sequential.cpp:183-213)
  __device__ int gca(const uint8_t* a, uint32_t na) {
    const uint32_t m = min(na, seqlen);
    uint32_t first = 0xffffffffu;
    for (uint32_t j0 = 0; j0 < m; j0 += 32) {
      const uint32_t j = j0 + lane;
      const bool d = j < m && a[j] != S.seq[j];
      const uint32_t b = __ballot_sync(GCL_FULL, d);
      if (b) {
        first = j0 + (uint32_t)(__ffs(b) - 1);
        break;
      }
    }
    return first == 0xffffffffu ? -1 : (int)first + 1;
  }

  // aut[label[j]] = elem[j] with the stored leaf given by its positions
  // (sequential.cpp:505-520, 544-555), written to ring slot num_aut % max_aut
  __device__ bool store_aut(const uint32_t (&pos)[VPL]) {
    const uint32_t idx = (uint32_t)num_aut % A.max_aut;
    if (idx >= A.aut_cap) {
      status = kAutOverflow;
      return false;
    }
#pragma unroll
    for (int k = 0; k < VPL; ++k)
      if (valid(k)) S.map[L.cs[k]] = (uint8_t)vid(k);  // position -> vertex
    __syncwarp();
    uint8_t* dst = auts + (uint64_t)idx * 64u;
#pragma unroll
    for (int k = 0; k < VPL; ++k)
      if (valid(k)) dst[vid(k)] = S.map[pos[k]];
    __syncwarp();
    ++num_aut;
    return true;
  }

  // ---- orbits of the stored automorphisms fixing the current sequence
  //      (perm_group.cpp:5-116) ------------------------------------------
  // Root of x: parents only point to smaller vertices, so at most n steps.
  __device__ uint32_t find(uint32_t x) {
    volatile uint32_t* d = S.dsu;
    uint32_t p = d[x];
    for (int step = 0; p != x && p < x && step < kW64MaxN; ++step) {
      x = p;
      p = d[x];
    }
    return x;
  }

  __device__ void orbits(int idx) {
    const int limit = num_aut < (int)A.max_aut ? num_aut : (int)A.max_aut;
    int from = S.tc[idx].last;
    if (from == -1) from = 0;
    const uint64_t mem = S.tc[idx].members;
    const bool rv = S.tc[idx].reps_valid;
    uint8_t* rp = reps + (uint64_t)idx * 64u;
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      if (!valid(k)) continue;
      const uint32_t v = vid(k);
      S.dsu[v] = ((mem >> v) & 1ull) ? (rv ? (uint32_t)rp[v] : v) : v;
    }
    __syncwarp();
    bool any = false;
    for (int i = from; i < limit; ++i) {
      const uint8_t* pm = auts + (uint64_t)i * 64u;
      bool bad = false;
      for (uint32_t j = lane; j < seqlen; j += 32) {
        const uint32_t sv = S.seq[j];
        if (pm[sv] != sv) bad = true;
      }
      if (__any_sync(GCL_FULL, bad)) continue;
      any = true;
      uint32_t img[VPL];
#pragma unroll
      for (int k = 0; k < VPL; ++k) img[k] = valid(k) ? pm[vid(k)] : vid(k);
      // union every (v, pm[v]) with min-root hooking until no edge is left
      // between two roots; a root is always the minimum of its tree.  Each
      // round merges at least two trees, so n rounds always suffice.
      for (int round = 0;; ++round) {
        if (round > kW64MaxN + 1) {
          fail(kInternal);
          return;
        }
        bool changed = false;
#pragma unroll
        for (int k = 0; k < VPL; ++k) {
          if (!valid(k) || img[k] == vid(k)) continue;
          const uint32_t a = find(vid(k)), b = find(img[k]);
          if (a != b) {
            atomicMin(&S.dsu[max(a, b)], min(a, b));
            changed = true;
          }
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < VPL; ++k)
          if (valid(k)) {
            const uint32_t r = find(vid(k));
            atomicMin(&S.dsu[vid(k)], r);
          }
        __syncwarp();
        if (!__any_sync(GCL_FULL, changed)) break;
      }
    }
    if (!any) return;
    bool isrep[VPL];
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      isrep[k] = false;
      if (!valid(k)) continue;
      const uint32_t v = vid(k);
      if ((mem >> v) & 1ull) {
        const uint32_t r = find(v);
        rp[v] = (uint8_t)r;
        isrep[k] = r == v;
      }
    }
    const uint64_t rm = ballot64<VPL>(isrep);
    __syncwarp();
    if (lane == 0) {
      S.tc[idx].repmask = rm;
      S.tc[idx].reps_valid = 1;
    }
    __syncwarp();
  }

  // ---- first_terminal (sequential.cpp:259-303) ---------------------------
  __device__ void first_terminal() {
    uint64_t R[VPL];
    leaf_rows(R);
    eqlevfirst = level;
#pragma unroll
    for (int k = 0; k < VPL; ++k) {
      if (!valid(k)) continue;
      S.first_cert[L.cs[k]] = R[k];
      S.best_cert[L.cs[k]] = R[k];
      L.fpos[k] = L.bpos[k] = L.cs[k];
    }
    for (uint32_t j = lane; j < seqlen; j += 32) S.first_seq[j] = S.best_seq[j] = S.seq[j];
    for (uint32_t j = lane; j < level; j += 32) S.canoncode[j] = S.firstcode[j];
    __syncwarp();
    if (lane == 0) {
      S.firstcode[level] = (uint16_t)kSentinel;
      S.canoncode[level] = (uint16_t)kSentinel;
    }
    __syncwarp();
    first_seqlen = best_seqlen = seqlen;
    first_found = true;
    canon_level = eqlevcanon = (int)level;
    comp_canon = 0;
  }

  __device__ void first_path_node() {
    if (discrete()) {
      first_terminal();
      backtrack(level - 1);
      return;
    }
    select_tc();
    if (status != kOk) return;
    const int idx = tcl - 1;
    next_rep(idx);
    push_and_split(idx);
    if (status != kOk) return;
    if (lane == 0) S.firstcode[level - 1] = (uint16_t)code;
    __syncwarp();
  }

  // ---- classify_node (sequential.cpp:396-624) ----------------------------
  __device__ bool classify() {
    const uint32_t Lv = level;
    if (eqlevfirst == Lv - 1 && code == (int)S.firstcode[Lv - 1]) eqlevfirst = Lv;
    if (eqlevcanon == (int)Lv - 1) {
      const int cc = S.canoncode[Lv - 1];
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
      if (lane == 0) S.canoncode[Lv - 1] = (uint16_t)code;
      __syncwarp();
    }
    int dec = 0;
    uint64_t R[VPL];
    if (eqlevfirst != Lv && comp_canon < 0) {
      dec = 4;
    } else if (discrete()) {
      leaf_rows(R);
      if (eqlevfirst == Lv && rows_equal(R, S.first_cert)) dec = 1;
      if (dec == 0) {
        if (comp_canon == 0) {
          if ((int)Lv < canon_level)
            comp_canon = 1;
          else
            comp_canon = cmp_upper(R, S.best_cert);
        }
        dec = comp_canon == 0 ? 2 : (comp_canon > 0 ? 3 : 4);
      }
    }
    switch (dec) {
      case 1: {
        if (!store_aut(L.fpos)) return false;
        const int g = gca(S.first_seq, first_seqlen);
        backtrack(g >= 0 ? (uint32_t)g : Lv - 1);
        break;
      }
      case 2: {
        if (!store_aut(L.bpos)) return false;
        const int g = gca(S.best_seq, best_seqlen);
        backtrack(g >= 0 ? (uint32_t)g : Lv - 1);
        break;
      }
      case 3: {
        canon_level = eqlevcanon = (int)Lv;
        comp_canon = 0;
        store_rows(R, S.best_cert);
#pragma unroll
        for (int k = 0; k < VPL; ++k) L.bpos[k] = L.cs[k];
        copy_seq(S.best_seq);
        if (lane == 0) S.canoncode[Lv] = (uint16_t)kSentinel;
        __syncwarp();
        best_seqlen = seqlen;
        backtrack(Lv - 1);
        break;
      }
      case 4:
        backtrack(Lv - 1);
        break;
      default:
        break;
    }
    return true;
  }

  // ---- other_path_node (sequential.cpp:304-392) ---------------------------
  __device__ bool other_path_node() {
    if (!discrete() && (eqlevfirst == level || comp_canon >= 0)) {
      if (tcl < (int)level) select_tc();
      if (status != kOk) return false;
      const int idx = (int)level - 1;
      if (S.tc[idx].counter >= (uint32_t)n) {
        backtrack(level - 1);
        return true;
      }
      if (num_aut > 0 && num_aut > S.tc[idx].last) {
        orbits(idx);
        if (status != kOk) return false;
        __syncwarp();
        if (lane == 0) S.tc[idx].last = num_aut;
        __syncwarp();
      }
      if (!next_rep(idx)) {
        backtrack(level - 1);
        return true;
      }
      push_and_split(idx);
      if (status != kOk) return false;
    }
    return classify();
  }

  // ---- search_tree_traversal (sequential.cpp:626-648) ---------------------
  __device__ void run() {
    code = refine(starts);
    if (status != kOk) return;
    if (lane == 0) S.firstcode[level - 1] = (uint16_t)code;
    __syncwarp();
    nodes = 1;
    while (level >= 1 && status == kOk) {
      if ((nodes & 63) == 0 && out_of_time()) {
        fail(kTimeout);
        break;
      }
      if (!first_found) {
        first_path_node();
      } else if (!other_path_node()) {
        return;  // overflow of the automorphism ring or a failed check
      }
    }
  }
};

template <int VPL>
__device__ void w64_canon_one(W64Smem& S, const BatchArgs& A, int g, uint8_t* slot) {
  const int64_t vo = A.voff[g];
  const int n = (int)(A.voff[g + 1] - vo);
  W64Search<VPL> W(S, A, n, slot);
  const uint32_t lane = W.lane;
  if (A.budget_ns) W.deadline = __shfl_sync(GCL_FULL, lane == 0 ? global_ns() : 0ull, 0) + A.budget_ns;
  if (!W.load(vo, A.rowptr + vo + g, A.col + A.eoff[g], A.color, A.eoff[g + 1] - A.eoff[g])) {
    if (lane == 0) A.status[g] = kBadInput;
    return;
  }
  W.run();
  if (lane == 0) {
    A.status[g] = W.status;
    if (A.out_stats) {
      A.out_stats[2 * (int64_t)g] = W.num_aut;
      A.out_stats[2 * (int64_t)g + 1] = W.nodes;
    }
  }
  if (W.status != kOk) return;
  // canonical labeling: position -> vertex of the best leaf
  if (A.out_label) {
#pragma unroll
    for (int k = 0; k < VPL; ++k)
      if (W.valid(k)) A.out_label[vo + W.L.bpos[k]] = (int32_t)W.vid(k);
  }
  if (A.out_cert) {
    for (int p = lane; p < n; p += 32) A.out_cert[vo + p] = S.best_cert[p];
  }
  if (A.out_dense) {
    uint8_t* o = A.out_dense + A.ooff[g];
    const int nn = n * n;
    for (int i = lane; i < nn; i += 32) {
      const int r = i / n, c = i - r * n;
      o[i] = (uint8_t)((S.best_cert[r] >> c) & 1ull);
    }
  }
}

}  // namespace gcl
