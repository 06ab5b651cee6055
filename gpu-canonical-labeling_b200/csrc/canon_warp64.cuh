// canon_warp64.cuh -- one warp canonizes one graph with n <= 64 vertices.
//
// The search is the reference's sequential individualization-refinement DFS
// (src/sequential.cpp:216-670) step for step, so the canonical form, the
// number of stored automorphisms and the number of search-tree nodes equal
// the reference's on every input.  What changes is the representation:
//
//   * a vertex set is one 64-bit mask; lane L owns vertices L and L+32 and
//     positions L and L+32;
//   * the ordered partition is vertex-indexed: each vertex knows the start
//     position `cs` of its cell, each cell start knows the member mask of its
//     cell, and the warp holds `starts`, the mask of cell start positions.  The
//     order of vertices inside a cell is never stored: the reference's
//     refinement and search depend only on the cells as sets (fragments are
//     ordered by count, targets and branch vertices are chosen by position and
//     by vertex id), so leaves, codes and pruning decisions are unchanged;
//   * counting neighbours in a splitter is popc(adj[v] & splitter); splitting
//     every cell at once is a radix pass over the count bits with warp
//     ballots; only the invariant hash (a serial, order-dependent chain) is
//     folded over a mask of hash items in position order;
//   * a leaf certificate is one 64-bit row per canonical vertex; the
//     reference's n^2 upper-triangle compare (sequential.cpp:114-124) becomes
//     a masked row compare plus a warp min, and the isAutomorphism test
//     against the first leaf (sequential.cpp:127-167) becomes certificate
//     equality, which is the same predicate for a bijection.
//
// Code layout: the warp's state lives in shared memory between phases.  The
// root step (load and root refinement), the search below the root, the root
// hand-over and the output writer are non-inlined functions, so an SM's warps
// share a small instruction footprint across those stages; the per-node
// phases (refine, individualize, backtrack, orbits, leaf work) are inlined
// into them.  Timed on the batched small-graph workload: inlining the
// per-node phases cut the pipelined launch by 13% (calls cost register
// saves and restores through local memory on every node), while inlining the
// root step or the whole search as well made it slower again.
#pragma once
#include <cstdint>

#include "gcl_device.cuh"

namespace gcl {

constexpr int kW64MaxN = 64;
constexpr int kW64Levels = kW64MaxN + 2;
constexpr int kW64Threads = 128;  // 4 warps per block, one graph per warp
constexpr int kW64Warps = kW64Threads / 32;
constexpr int kW64AutHead = 8;  // first ring entries kept in shared memory

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
  uint64_t adj[kW64MaxN];         // vertex -> neighbour mask
  uint64_t cmask[kW64MaxN];       // cell start position -> member mask
  uint64_t first_cert[kW64MaxN];  // first leaf, one row per canonical vertex
  uint64_t best_cert[kW64MaxN];   // best leaf
  TcHdr tc[kW64Levels];
  uint32_t dsu[kW64MaxN];
  uint16_t firstcode[kW64Levels];
  uint16_t canoncode[kW64Levels];
  uint8_t cs[kW64MaxN];     // vertex -> start position of its cell
  uint8_t inlev[kW64MaxN];  // cell start position -> in_level
  uint8_t fk[kW64MaxN];     // fragment start position -> its neighbour count
  uint8_t seq[kW64MaxN];
  uint8_t first_seq[kW64MaxN];
  uint8_t best_seq[kW64MaxN];
  uint8_t fpos[kW64MaxN];  // vertex -> position in the first leaf
  uint8_t bpos[kW64MaxN];  // vertex -> position in the best leaf
  uint8_t map[kW64MaxN];
  uint8_t pv[kW64MaxN];  // singleton cell start position -> its vertex
  uint64_t sing;         // vertices whose cell is a singleton
  // ring entries 0..kW64AutHead-1 and their fixed-point masks; later entries
  // live in the slot workspace
  uint8_t aut_head[kW64AutHead][kW64MaxN];
  uint64_t fix_head[kW64AutHead];
};

// One W64Smem per warp of the block, at namespace scope so every phase
// function addresses it directly in the shared window.
__shared__ W64Smem g_w64[kW64Warps];

__device__ __forceinline__ W64Smem& w64_smem() { return g_w64[threadIdx.x >> 5]; }

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
  uint64_t* out_rows;    // packed rows per graph at roff[g], or null
  const int64_t* roff;   // ceil(n/64) words per row, n rows per graph
  int32_t* out_label;    // n per graph at voff[g], or null
  int64_t* out_stats;    // {num_aut, nodes} per graph, or null
  int32_t* status;       // per graph
  uint8_t* work;         // per-warp slot workspace
  uint64_t slot_bytes;
  uint64_t budget_ns;    // per-graph time budget (0 = unlimited)
};

// Per-slot workspace layout: reps[kW64Levels][64], the automorphism ring
// (aut_cap x 64 bytes), then one fixed-point mask per ring entry (aut_cap x
// 8 bytes).  The first kW64AutHead entries of both are used from shared
// memory instead.
__host__ __device__ constexpr uint64_t w64_slot_bytes(uint32_t aut_cap) {
  return ((uint64_t)kW64Levels * 64u + (uint64_t)aut_cap * 72u + 255u) & ~255ull;
}

__device__ __forceinline__ uint64_t ballot2(bool a, bool b) {
  return (uint64_t)__ballot_sync(GCL_FULL, a) | ((uint64_t)__ballot_sync(GCL_FULL, b) << 32);
}
__device__ __forceinline__ uint64_t bit64(uint32_t p) { return 1ull << p; }

// ---------------------------------------------------------------------------
// Partition_s_refinement (partition_refinement.cpp:150-485).
// `active` holds the start positions of the initially active cells.  Returns
// the new starts mask and the refinement code (the caller increments level).
// ---------------------------------------------------------------------------
struct W64Refined {
  uint64_t starts;
  int code;
  int ok;
};

static __device__ __forceinline__ W64Refined w64_refine(int n, uint64_t starts, uint32_t level,
                                                     uint64_t active) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  const uint64_t full = low_mask((uint32_t)n);
  const uint32_t v0 = lane, v1 = lane + 32;
  const bool ok0 = v0 < (uint32_t)n, ok1 = v1 < (uint32_t)n;
  const uint64_t adj0 = ok0 ? S.adj[v0] : 0ull, adj1 = ok1 ? S.adj[v1] : 0ull;
  const uint32_t lvl1 = level + 1;
  const uint64_t lastbit = bit64((uint32_t)n - 1);
  uint64_t sing = S.sing;
  uint32_t lc = popc64(starts), hint = 0, iters = 0;
  int ok = 1;
  // registers: the member masks of the cells starting at positions lane and
  // lane + 32 (valid where `starts` has the bit), and the cells of vertices
  // lane and lane + 32
  uint64_t cmr0 = S.cmask[v0], cmr1 = S.cmask[v1];
  uint32_t csr0 = ok0 ? S.cs[v0] : 0u, csr1 = ok1 ? S.cs[v1] : 0u;
  while (starts != full && active) {
    if (++iters > 64u * 64u + 64u) {  // every step removes an active cell or splits one
      ok = 0;
      break;
    }
    // splitter: hint if active, else the next active after it, else wrap
    uint32_t s;
    if ((active >> hint) & 1ull) {
      s = hint;
    } else {
      const uint64_t a = active & ge_mask(hint + 1);
      s = ctz64(a ? a : active);
    }
    active &= ~bit64(s);
    const uint64_t nx = starts & ge_mask(s + 1);
    const uint32_t e = nx ? ctz64(nx) : (uint32_t)n;
    lc = mash(lc, s + e - 1);  // split1 + split2
    if (e - s == 1) {
      // Singleton splitter {w}: a cell splits into [neighbours, non-neighbours]
      // when N(w) meets it partially.  Only neighbours outside singleton
      // cells can be in such a cell, so most steps end here.
      const uint64_t N = S.adj[S.pv[s]];
      const uint64_t X = N & ~sing;
      if (!X) continue;
      // a cell splits when N meets it partially: the lanes test the cells
      // starting at their two positions
      const bool sp0 = ((starts >> v0) & 1ull) && (cmr0 & N) && (cmr0 & ~N);
      const bool sp1 = ((starts >> v1) & 1ull) && (cmr1 & N) && (cmr1 & ~N);
      const uint64_t splitc = ballot2(sp0, sp1);
      if (!splitc) continue;
      // The split cells, each by the lane owning its start (:296-465): the
      // neighbours keep the start c, the rest start at p = c + |C & N|.
      // Cells are disjoint ranges, and whether c was active does not depend
      // on the cells before it, so they split independently; only the hash
      // and the hint follow position order (below).
      uint64_t addA = 0, addS = 0, addG = 0;  // active, starts, singleton additions
      uint32_t hv0 = 0xffu, hv1 = 0xffu, nbp = 0;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        if (!(k ? sp1 : sp0)) continue;
        const uint32_t c = k ? v1 : v0;
        const uint64_t C = k ? cmr1 : cmr0, CN = C & N, CR = C & ~N;
        const uint32_t nb = popc64(CN), nn = popc64(CR), p = c + nb;
        uint32_t hv = 0xffu;
        if (((active >> c) & 1ull) || nb >= nn) {
          addA |= bit64(p);
          if (nn == 1) hv = p;
        } else {
          addA |= bit64(c);
          if (nb == 1) hv = c;
        }
        addS |= bit64(p);
        if (nb == 1) addG |= CN;
        if (nn == 1) addG |= CR;
        S.cmask[c] = CN;
        S.cmask[p] = CR;
        S.inlev[p] = S.inlev[c];
        S.inlev[c] = (uint8_t)lvl1;
        if (nb == 1) S.pv[c] = (uint8_t)ctz64(CN);
        if (nn == 1) S.pv[p] = (uint8_t)ctz64(CR);
        if (k) {
          cmr1 = CN;
          hv1 = hv;
          nbp |= nb << 8;
        } else {
          cmr0 = CN;
          hv0 = hv;
          nbp |= nb;
        }
      }
      // hash: cell.first + neighbors_size - 1 per split cell, in position order
      for (uint64_t t = splitc; t; t &= t - 1) {
        const uint32_t c = ctz64(t);
        const uint32_t w = __shfl_sync(GCL_FULL, nbp, (int)(c & 31u));
        lc = mash(lc, c + ((c >= 32u ? w >> 8 : w) & 0xffu) - 1u);
      }
      // hint: the last split cell in position order that sets one
      const uint64_t hc = ballot2(hv0 != 0xffu, hv1 != 0xffu);
      if (hc) {
        const uint32_t cl = msb64(hc);
        hint = __shfl_sync(GCL_FULL, cl >= 32u ? hv1 : hv0, (int)(cl & 31u));
      }
      active |= warp_or64(addA);
      const uint64_t NSt = warp_or64(addS);
      starts |= NSt;
      sing |= warp_or64(addG);
      // vertices of split cells outside N move to the second fragment
      {
        const uint32_t w0 = __shfl_sync(GCL_FULL, nbp, (int)(csr0 & 31u));
        const uint32_t w1 = __shfl_sync(GCL_FULL, nbp, (int)(csr1 & 31u));
        if (ok0 && ((splitc >> csr0) & 1ull) && !((N >> v0) & 1ull)) {
          csr0 += (csr0 >= 32u ? w0 >> 8 : w0) & 0xffu;
          S.cs[v0] = (uint8_t)csr0;
        }
        if (ok1 && ((splitc >> csr1) & 1ull) && !((N >> v1) & 1ull)) {
          csr1 += (csr1 >= 32u ? w1 >> 8 : w1) & 0xffu;
          S.cs[v1] = (uint8_t)csr1;
        }
      }
      __syncwarp();
      // the new fragments' member masks, written by their cells' owners
      if ((NSt >> v0) & 1ull) cmr0 = S.cmask[v0];
      if ((NSt >> v1) & 1ull) cmr1 = S.cmask[v1];
    } else {
      // Non-singleton splitter: fragments in ascending neighbour count.
      lc = mash(lc, e - s);
      const uint64_t spl = S.cmask[s];
      uint32_t cs0 = csr0, cs1 = csr1;
      uint64_t cm0 = ok0 ? S.cmask[cs0] : 0ull, cm1 = ok1 ? S.cmask[cs1] : 0ull;
      const uint32_t k0 = ok0 ? popc64(adj0 & spl) : 0u, k1 = ok1 ? popc64(adj1 & spl) : 0u;
      const uint32_t mx = __reduce_max_sync(GCL_FULL, max(k0, k1));
      uint32_t lt0 = 0, lt1 = 0;
      for (int b = mx ? 31 - __clz((int)mx) : -1; b >= 0; --b) {
        const bool b0 = (k0 >> b) & 1u, b1 = (k1 >> b) & 1u;
        const uint64_t M = ballot2(b0, b1);
        if (b0) {
          lt0 += popc64(cm0 & ~M);
          cm0 &= M;
        } else {
          cm0 &= ~M;
        }
        if (b1) {
          lt1 += popc64(cm1 & ~M);
          cm1 &= M;
        } else {
          cm1 &= ~M;
        }
      }
      cs0 += lt0;
      cs1 += lt1;
      const uint64_t ns = (ok0 ? bit64(cs0) : 0ull) | (ok1 ? bit64(cs1) : 0ull);
      const bool s0 = ok0 && popc64(cm0) == 1, s1 = ok1 && popc64(cm1) == 1;
      sing = ballot2(s0, s1);
      __syncwarp();  // every lane has read the old cell masks
      if (ok0) {
        S.cs[v0] = (uint8_t)cs0;
        S.cmask[cs0] = cm0;
        S.fk[cs0] = (uint8_t)k0;
        if (s0) S.pv[cs0] = (uint8_t)v0;
      }
      if (ok1) {
        S.cs[v1] = (uint8_t)cs1;
        S.cmask[cs1] = cm1;
        S.fk[cs1] = (uint8_t)k1;
        if (s1) S.pv[cs1] = (uint8_t)v1;
      }
      const uint64_t NS = warp_or64(ns) & ~starts;
      __syncwarp();
      // hash items in position order: every start of a non-singleton old
      // cell (common count) and every new fragment start (:253-373)
      const uint64_t singles = starts & ((starts >> 1) | lastbit);
      uint64_t t = (starts & ~singles) | NS;
      while (t) {
        const uint32_t p = ctz64(t);
        t &= t - 1;
        lc = mash(lc, (uint32_t)S.fk[p] + p);
      }
      if (NS) {
        const uint64_t all = starts | NS;
        // in_level of the fragments of split cells: level+1, the last one
        // keeps the cell's old in_level (:342, 463-465)
        uint32_t w0 = 0xffu, w1 = 0xffu;
        if ((all >> v0) & 1ull) {
          const uint32_t c = msb64(starts & low_mask(v0 + 1));
          const uint64_t nc = starts & ge_mask(c + 1);
          const uint32_t end = nc ? ctz64(nc) : (uint32_t)n;
          if (NS & low_mask(end) & ge_mask(c + 1))
            w0 = (v0 == msb64(all & low_mask(end))) ? S.inlev[c] : lvl1;
        }
        if ((all >> v1) & 1ull) {
          const uint32_t c = msb64(starts & low_mask(v1 + 1));
          const uint64_t nc = starts & ge_mask(c + 1);
          const uint32_t end = nc ? ctz64(nc) : (uint32_t)n;
          if (NS & low_mask(end) & ge_mask(c + 1))
            w1 = (v1 == msb64(all & low_mask(end))) ? S.inlev[c] : lvl1;
        }
        // active set (:436-460): every new fragment; for a cell that was not
        // active, its first fragment in and its first largest fragment out.
        // hint: the last new singleton fragment in position order.
        const uint64_t single_all = all & ((all >> 1) | lastbit);
        const uint64_t hs = NS & single_all;
        if (hs) hint = msb64(hs);
        // each fragment start of a split cell that was not active offers
        // (size, -position) for its cell's first largest fragment, one
        // shared-memory max per cell (S.dsu is free outside the orbits)
        uint32_t key0 = 0, key1 = 0, cell0 = 0, cell1 = 0;
        bool fr0 = false, fr1 = false;
        if ((all >> v0) & 1ull) {
          cell0 = msb64(starts & low_mask(v0 + 1));
          const uint64_t nc = starts & ge_mask(cell0 + 1);
          const uint32_t end = nc ? ctz64(nc) : (uint32_t)n;
          const uint64_t nf = all & ge_mask(v0 + 1);
          fr0 = !((active >> cell0) & 1ull) && (NS & low_mask(end) & ge_mask(cell0 + 1)) != 0;
          key0 = ((min(nf ? ctz64(nf) : (uint32_t)n, end) - v0) << 6) | (63u - v0);
        }
        if ((all >> v1) & 1ull) {
          cell1 = msb64(starts & low_mask(v1 + 1));
          const uint64_t nc = starts & ge_mask(cell1 + 1);
          const uint32_t end = nc ? ctz64(nc) : (uint32_t)n;
          const uint64_t nf = all & ge_mask(v1 + 1);
          fr1 = !((active >> cell1) & 1ull) && (NS & low_mask(end) & ge_mask(cell1 + 1)) != 0;
          key1 = ((min(nf ? ctz64(nf) : (uint32_t)n, end) - v1) << 6) | (63u - v1);
        }
        __syncwarp();
        if (fr0 && cell0 == v0) S.dsu[cell0] = 0;
        if (fr1 && cell1 == v1) S.dsu[cell1] = 0;
        __syncwarp();
        if (fr0) atomicMax(&S.dsu[cell0], key0);
        if (fr1) atomicMax(&S.dsu[cell1], key1);
        __syncwarp();
        const uint64_t out = ballot2(fr0 && S.dsu[cell0] == key0, fr1 && S.dsu[cell1] == key1);
        const uint64_t in = ballot2(fr0 && cell0 == v0, fr1 && cell1 == v1);
        active = (active | NS | in) & ~out;
        __syncwarp();
        if (w0 != 0xffu) S.inlev[v0] = (uint8_t)w0;
        if (w1 != 0xffu) S.inlev[v1] = (uint8_t)w1;
        starts = all;
      }
      __syncwarp();
      csr0 = cs0;
      csr1 = cs1;
      cmr0 = S.cmask[v0];
      cmr1 = S.cmask[v1];
    }
  }
  __syncwarp();
  if (lane == 0) S.sing = sing;
  __syncwarp();
  return {starts, cleanup(mash(lc, popc64(starts))), ok};
}

// split_by_and_refine's split (partition_refinement.cpp:486-528): vertex v
// moves to a singleton cell at t, the rest of the cell starts at t+1.
// Returns false when the cell is already a singleton (nothing to refine).
static __device__ __forceinline__ bool w64_individualize(int n, uint32_t level, uint32_t v, uint32_t t) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  const uint64_t mem = S.cmask[t];
  if (popc64(mem) <= 1) return false;
  const uint32_t v0 = lane, v1 = lane + 32;
  __syncwarp();
  if (v0 < (uint32_t)n && ((mem >> v0) & 1ull) && v0 != v) S.cs[v0] = (uint8_t)(t + 1);
  if (v1 < (uint32_t)n && ((mem >> v1) & 1ull) && v1 != v) S.cs[v1] = (uint8_t)(t + 1);
  if (lane == 0) {
    const uint64_t rest = mem & ~bit64(v);
    S.cmask[t] = bit64(v);
    S.cmask[t + 1] = rest;
    S.inlev[t + 1] = S.inlev[t];
    S.inlev[t] = (uint8_t)(level + 1);
    S.pv[t] = (uint8_t)v;
    uint64_t sg = S.sing | bit64(v);
    if (popc64(rest) == 1) {
      sg |= rest;
      S.pv[t + 1] = (uint8_t)ctz64(rest);
    }
    S.sing = sg;
  }
  __syncwarp();
  return true;
}

// reconstruct_at_level (partition_refinement.cpp:541-604): every maximal run
// of cells created after level Lv merges with the cell that follows it, and
// the merged cell takes that cell's in_level.  Returns the new starts mask
// (0 if the partition is inconsistent).
static __device__ __forceinline__ uint64_t w64_backtrack(int n, uint64_t starts, uint32_t Lv) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  const uint32_t q0 = lane, q1 = lane + 32;
  const bool st0 = q0 < (uint32_t)n && ((starts >> q0) & 1ull);
  const bool st1 = q1 < (uint32_t)n && ((starts >> q1) & 1ull);
  const bool big0 = st0 && S.inlev[q0] > Lv, big1 = st1 && S.inlev[q1] > Lv;
  const uint64_t BIG = ballot2(big0, big1);
  if (!BIG) return starts;
  bool sv0 = st0, sv1 = st1;
  if (st0 && q0 > 0 && ((BIG >> msb64(starts & low_mask(q0))) & 1ull)) sv0 = false;
  if (st1 && ((BIG >> msb64(starts & low_mask(q1))) & 1ull)) sv1 = false;
  const uint64_t NST = ballot2(sv0, sv1);
  uint32_t nl0 = 0, nl1 = 0;
  uint64_t m0 = 0, m1 = 0;
  bool bad = false, w0 = false, w1 = false;
  if (sv0 && big0) {
    const uint64_t j = starts & ~BIG & ge_mask(q0 + 1);
    if (!j) bad = true;
    else nl0 = S.inlev[ctz64(j)];
    const uint64_t nn = NST & ge_mask(q0 + 1);
    uint64_t r = starts & ge_mask(q0) & low_mask(nn ? ctz64(nn) : (uint32_t)n);
    while (r) {
      m0 |= S.cmask[ctz64(r)];
      r &= r - 1;
    }
    w0 = true;
  }
  if (sv1 && big1) {
    const uint64_t j = starts & ~BIG & ge_mask(q1 + 1);
    if (!j) bad = true;
    else nl1 = S.inlev[ctz64(j)];
    const uint64_t nn = NST & ge_mask(q1 + 1);
    uint64_t r = starts & ge_mask(q1) & low_mask(nn ? ctz64(nn) : (uint32_t)n);
    while (r) {
      m1 |= S.cmask[ctz64(r)];
      r &= r - 1;
    }
    w1 = true;
  }
  if (__any_sync(GCL_FULL, bad)) return 0;
  __syncwarp();
  if (w0) {
    S.inlev[q0] = (uint8_t)nl0;
    S.cmask[q0] = m0;
  }
  if (w1) {
    S.inlev[q1] = (uint8_t)nl1;
    S.cmask[q1] = m1;
  }
  uint32_t c0 = 0, c1 = 0;
  if (q0 < (uint32_t)n) {
    c0 = msb64(NST & low_mask((uint32_t)S.cs[q0] + 1));
    S.cs[q0] = (uint8_t)c0;
  }
  if (q1 < (uint32_t)n) {
    c1 = msb64(NST & low_mask((uint32_t)S.cs[q1] + 1));
    S.cs[q1] = (uint8_t)c1;
  }
  __syncwarp();
  // vertices in singleton cells after the merge; their pv entries are
  // unchanged (merging never creates a singleton)
  const bool g0 = q0 < (uint32_t)n && popc64(S.cmask[c0]) == 1;
  const bool g1 = q1 < (uint32_t)n && popc64(S.cmask[c1]) == 1;
  const uint64_t sg = ballot2(g0, g1);
  if (lane == 0) S.sing = sg;
  __syncwarp();
  return NST;
}

// Certificate rows of the lane's two vertices in a discrete partition: the
// neighbours renamed to positions (buildPermutedFlatAdjacencyMatrixArray,
// CSRGraph.cpp:332-351).  Row of vertex v belongs to canonical vertex cs[v].
struct Rows2 {
  uint64_t r0, r1;
};

static __device__ __forceinline__ Rows2 w64_leaf_rows(int n) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  Rows2 R{0ull, 0ull};
  if (lane < (uint32_t)n) {
    uint64_t a = S.adj[lane];
    while (a) {
      R.r0 |= bit64(S.cs[ctz64(a)]);
      a &= a - 1;
    }
  }
  if (lane + 32 < (uint32_t)n) {
    uint64_t a = S.adj[lane + 32];
    while (a) {
      R.r1 |= bit64(S.cs[ctz64(a)]);
      a &= a - 1;
    }
  }
  return R;
}

// compare_adj_upper(current, stored) (sequential.cpp:114-124)
static __device__ __forceinline__ int w64_cmp_upper(int n, Rows2 R, const uint64_t* B) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  uint32_t row = 64u;
  bool s0 = false, s1 = false;
  uint32_t p0 = 64u, p1 = 64u;
  if (lane < (uint32_t)n) {
    p0 = S.cs[lane];
    const uint64_t d = (R.r0 ^ B[p0]) & ge_mask(p0 + 1);
    if (d) {
      row = p0;
      s0 = (R.r0 >> ctz64(d)) & 1ull;
    }
  }
  if (lane + 32 < (uint32_t)n) {
    p1 = S.cs[lane + 32];
    const uint64_t d = (R.r1 ^ B[p1]) & ge_mask(p1 + 1);
    if (d) {
      row = min(row, p1);
      s1 = (R.r1 >> ctz64(d)) & 1ull;
    }
  }
  const uint32_t mrow = __reduce_min_sync(GCL_FULL, row);
  if (mrow == 64u) return 0;
  return ballot2(p0 == mrow && s0, p1 == mrow && s1) ? 1 : -1;
}

__device__ __forceinline__ bool w64_rows_equal(int n, Rows2 R, const uint64_t* B) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  const bool d0 = lane < (uint32_t)n && R.r0 != B[S.cs[lane]];
  const bool d1 = lane + 32 < (uint32_t)n && R.r1 != B[S.cs[lane + 32]];
  return ballot2(d0, d1) == 0;
}

// Rows into a stored certificate and the vertex positions into `pos`.
static __device__ __forceinline__ void w64_store_leaf(int n, Rows2 R, uint64_t* B, uint8_t* pos) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  __syncwarp();
  if (lane < (uint32_t)n) {
    B[S.cs[lane]] = R.r0;
    pos[lane] = S.cs[lane];
  }
  if (lane + 32 < (uint32_t)n) {
    B[S.cs[lane + 32]] = R.r1;
    pos[lane + 32] = S.cs[lane + 32];
  }
  __syncwarp();
}

// aut[label[j]] = elem[j] with the stored leaf given by its vertex positions
// (sequential.cpp:505-520, 544-555), written to one ring slot; its mask of
// fixed points goes to *fix.
static __device__ __forceinline__ void w64_store_aut(int n, const uint8_t* pos, uint8_t* dst,
                                                  uint64_t* fix) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  __syncwarp();
  if (lane < (uint32_t)n) S.map[S.cs[lane]] = (uint8_t)lane;  // position -> vertex
  if (lane + 32 < (uint32_t)n) S.map[S.cs[lane + 32]] = (uint8_t)(lane + 32);
  __syncwarp();
  bool f0 = false, f1 = false;
  if (lane < (uint32_t)n) {
    const uint8_t im = S.map[pos[lane]];
    dst[lane] = im;
    f0 = im == lane;
  }
  if (lane + 32 < (uint32_t)n) {
    const uint8_t im = S.map[pos[lane + 32]];
    dst[lane + 32] = im;
    f1 = im == lane + 32;
  }
  const uint64_t fm = ballot2(f0, f1);
  if (lane == 0) *fix = fm;
  __syncwarp();
}

// get_gca_level (sequential.cpp:183-213)
__device__ __forceinline__ int w64_gca(const uint8_t* a, uint32_t na, uint32_t seqlen) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  const uint32_t m = min(na, seqlen);
  const bool d0 = lane < m && a[lane] != S.seq[lane];
  const bool d1 = lane + 32 < m && a[lane + 32] != S.seq[lane + 32];
  const uint64_t b = ballot2(d0, d1);
  return b ? (int)ctz64(b) + 1 : -1;
}

// target_cell_selector (partition_refinement.cpp:607-655) with hint -1: the
// first non-singleton cell.
__device__ __forceinline__ void w64_select_tc(int n, uint64_t starts, int tcl) {
  W64Smem& S = w64_smem();
  const uint64_t singles = starts & ((starts >> 1) | bit64((uint32_t)n - 1));
  const uint32_t t = ctz64(starts & ~singles);
  const uint64_t mem = S.cmask[t];
  __syncwarp();
  if (lane_id() == 0) {
    TcHdr& h = S.tc[tcl];
    h.members = mem;
    h.repmask = mem;
    h.last = 0;
    h.counter = 0;
    h.first = (uint8_t)t;
    h.reps_valid = 0;
  }
  __syncwarp();
}

// subgroup_fixing_sequence + compute_orbits_fast (perm_group.cpp:5-116):
// orbits of the stored automorphisms that fix the current vertex sequence,
// merged into the target cell's previous orbits; each new representative is
// the least vertex of its merged orbit, as with the reference's min-root
// union-find.  A permutation fixes the sequence iff the sequence's vertex mask
// lies inside its fixed-point mask.  Such a permutation maps the target cell
// onto itself, so one that moves no member of the cell only joins vertices
// outside it and cannot change a member's orbit: only permutations that fix
// the sequence and move a member take part.
//
// The merge works on labels that are parent pointers to smaller vertices of
// the same component.  Every previous orbit is turned into one more
// permutation (a cycle through its members), so every edge of the union lies
// on a permutation cycle.  A round pulls the least label over all
// permutation images of a vertex (independent shared-memory loads), hooks the
// vertex's old parent under it (atomicMin), and shortcuts parents twice; a
// round that improves no label ends it, and then every vertex points at the
// least vertex of its component.  Returns false when the round bound was hit.
static __device__ __forceinline__ bool w64_orbits(int n, int idx, int num_aut, uint32_t max_aut,
                                               uint32_t seqlen, uint8_t* reps, const uint8_t* auts,
                                               const uint64_t* fixes) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  const int limit = num_aut < (int)max_aut ? num_aut : (int)max_aut;
  int from = S.tc[idx].last;
  if (from == -1) from = 0;
  const uint64_t mem = S.tc[idx].members;
  const uint64_t seqm = warp_or64((lane < seqlen ? bit64(S.seq[lane]) : 0ull) |
                                  (lane + 32 < seqlen ? bit64(S.seq[lane + 32]) : 0ull));
  // taking part: a bit per shared-memory head entry, and whether any later
  // (device-memory) entry does
  uint32_t selh = 0;
  bool seltail = false;
  for (int i = from; i < limit; ++i) {
    const uint64_t fm = i < kW64AutHead ? S.fix_head[i] : fixes[i];
    if ((seqm & ~fm) || !(mem & ~fm)) continue;
    if (i < kW64AutHead)
      selh |= 1u << i;
    else
      seltail = true;
  }
  if (!selh && !seltail) return true;  // no member's orbit can change
  const bool rv = S.tc[idx].reps_valid;
  uint8_t* rp = reps + (uint64_t)idx * 64u;
  const uint32_t v0 = lane, v1 = lane + 32;
  const bool ok0 = v0 < (uint32_t)n, ok1 = v1 < (uint32_t)n;
  uint32_t L0 = ok0 && ((mem >> v0) & 1ull) && rv ? (uint32_t)rp[v0] : v0;
  uint32_t L1 = ok1 && ((mem >> v1) & 1ull) && rv ? (uint32_t)rp[v1] : v1;
  // The orbits are the components of the graph whose edges join every
  // vertex v to its previous orbit's label L(v) and to its image under each
  // selected automorphism; a component is labelled by its least vertex.
  // Union-find with parent(v) = L(v) to start (L(v) <= v): lane l holds the
  // parents of vertices l and l + 32 packed in one word, so a lookup is one
  // shuffle; a hook (larger root under the smaller) is an atomicMin in
  // shared memory.  Parents never exceed their vertex, so every root is the
  // least vertex of its tree.
  uint32_t fp = (L0 & 0xffu) | ((L1 & 0xffu) << 8);
  uint32_t* par = S.dsu;
  // parent := grandparent until every vertex points at a root (a tree of
  // depth d needs ceil(log2 d) passes)
  auto compress = [&]() -> bool {
    for (int it = 0; it < 10; ++it) {
      const uint32_t f0 = fp & 0xffu, f1 = (fp >> 8) & 0xffu;
      const uint32_t g0 = __shfl_sync(GCL_FULL, fp, (int)(f0 & 31u));
      const uint32_t g1 = __shfl_sync(GCL_FULL, fp, (int)(f1 & 31u));
      const uint32_t h0 = (f0 >= 32u ? g0 >> 8 : g0) & 0xffu;
      const uint32_t h1 = (f1 >= 32u ? g1 >> 8 : g1) & 0xffu;
      const bool c = h0 != f0 || h1 != f1;
      fp = h0 | (h1 << 8);
      if (!__any_sync(GCL_FULL, c)) return true;
    }
    return false;
  };
  // the edges v -- pi(v) of one automorphism
  auto apply = [&](const uint8_t* img) -> bool {
    const uint32_t u0 = ok0 ? (uint32_t)img[v0] : v0, u1 = ok1 ? (uint32_t)img[v1] : v1;
    for (int round = 0; round <= kW64MaxN; ++round) {  // a hook round removes a root
      const uint32_t x0 = __shfl_sync(GCL_FULL, fp, (int)(u0 & 31u));
      const uint32_t x1 = __shfl_sync(GCL_FULL, fp, (int)(u1 & 31u));
      const uint32_t ra0 = fp & 0xffu, rb0 = (u0 >= 32u ? x0 >> 8 : x0) & 0xffu;
      const uint32_t ra1 = (fp >> 8) & 0xffu, rb1 = (u1 >= 32u ? x1 >> 8 : x1) & 0xffu;
      const bool d0 = ra0 != rb0, d1 = ra1 != rb1;
      if (!__any_sync(GCL_FULL, d0 || d1)) return true;
      par[v0] = ra0;
      par[v1] = ra1;
      __syncwarp();
      if (d0) atomicMin(&par[max(ra0, rb0)], min(ra0, rb0));
      if (d1) atomicMin(&par[max(ra1, rb1)], min(ra1, rb1));
      __syncwarp();
      fp = par[v0] | (par[v1] << 8);
      __syncwarp();  // read before the next round's stores
      if (!compress()) return false;
    }
    return false;
  };
  if (!compress()) return false;
#pragma unroll 1
  for (uint32_t k = 0; k < (uint32_t)kW64AutHead; ++k)
    if (((selh >> k) & 1u) && !apply(S.aut_head[k])) return false;
  if (seltail)
    for (int i = max(from, kW64AutHead); i < limit; ++i) {
      const uint64_t fm = fixes[i];
      if ((seqm & ~fm) || !(mem & ~fm)) continue;
      if (!apply(auts + (uint64_t)i * 64u)) return false;
    }
  L0 = fp & 0xffu;
  L1 = (fp >> 8) & 0xffu;
  bool r0 = false, r1 = false;
  if (ok0 && ((mem >> v0) & 1ull)) {
    rp[v0] = (uint8_t)L0;
    r0 = L0 == v0;
  }
  if (ok1 && ((mem >> v1) & 1ull)) {
    rp[v1] = (uint8_t)L1;
    r1 = L1 == v1;
  }
  const uint64_t rm = ballot2(r0, r1);
  __syncwarp();
  if (lane == 0) {
    S.tc[idx].repmask = rm;
    S.tc[idx].reps_valid = 1;
  }
  __syncwarp();
  return true;
}

// Adjacency masks and the colour partition (initializePartition_s,
// partition_refinement.cpp:28-68: cells are the colour classes in ascending
// colour order).  Returns the starts mask, or 0 for invalid input.
static __device__ __noinline__ uint64_t w64_load(int n, const int32_t* rp, const int32_t* cl,
                                          const int32_t* color, int64_t m) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  bool bad = false;
  uint64_t a0 = 0, a1 = 0;
  for (int k = 0; k < 2; ++k) {
    const uint32_t v = lane + 32u * k;
    if (v >= (uint32_t)n) continue;
    uint64_t a = 0;
    const int32_t b = rp[v], e = rp[v + 1];
    if (b < 0 || e < b || (int64_t)e > m) bad = true;
    for (int32_t i = b; i < e && !bad; ++i) {
      const int32_t u = cl[i];
      if (u < 0 || u >= n || (uint32_t)u == v || ((a >> u) & 1ull)) {
        bad = true;
        break;
      }
      a |= bit64((uint32_t)u);
    }
    S.adj[v] = a;
    if (k)
      a1 = a;
    else
      a0 = a;
  }
  __syncwarp();
  // both directions stored (CSRGraph::fromDIMACS inserts both)
  for (int k = 0; k < 2; ++k) {
    uint64_t a = k ? a1 : a0;
    const uint32_t v = lane + 32u * k;
    while (a && !bad) {
      if (!((S.adj[ctz64(a)] >> v) & 1ull)) bad = true;
      a &= a - 1;
    }
  }
  if (__any_sync(GCL_FULL, bad)) return 0;
  const int32_t c0 = (color && lane < (uint32_t)n) ? color[lane] : 0;
  const int32_t c1 = (color && lane + 32 < (uint32_t)n) ? color[lane + 32] : 0;
  uint64_t starts;
  if (!__any_sync(GCL_FULL, c0 != 0 || c1 != 0)) {
    if (lane < (uint32_t)n) S.cs[lane] = 0;
    if (lane + 32 < (uint32_t)n) S.cs[lane + 32] = 0;
    if (lane == 0) {
      S.cmask[0] = low_mask((uint32_t)n);
      S.pv[0] = 0;
      S.sing = n == 1 ? 1ull : 0ull;
    }
    starts = 1ull;
  } else {
    int32_t* ct = reinterpret_cast<int32_t*>(S.dsu);
    if (lane < (uint32_t)n) ct[lane] = c0;
    if (lane + 32 < (uint32_t)n) ct[lane + 32] = c1;
    __syncwarp();
    uint32_t b0 = 0, b1 = 0;
    uint64_t same0 = 0, same1 = 0;
    for (int u = 0; u < n; ++u) {
      const int32_t cu = ct[u];
      b0 += cu < c0;
      b1 += cu < c1;
      same0 |= (uint64_t)(cu == c0) << u;
      same1 |= (uint64_t)(cu == c1) << u;
    }
    uint64_t st = 0;
    __syncwarp();
    if (lane < (uint32_t)n) {
      S.cs[lane] = (uint8_t)b0;
      S.cmask[b0] = same0;
      st |= bit64(b0);
      if (popc64(same0) == 1) S.pv[b0] = (uint8_t)lane;
    }
    if (lane + 32 < (uint32_t)n) {
      S.cs[lane + 32] = (uint8_t)b1;
      S.cmask[b1] = same1;
      st |= bit64(b1);
      if (popc64(same1) == 1) S.pv[b1] = (uint8_t)(lane + 32);
    }
    starts = warp_or64(st);
    const uint64_t sg = ballot2(lane < (uint32_t)n && popc64(same0) == 1,
                                lane + 32 < (uint32_t)n && popc64(same1) == 1);
    if (lane == 0) S.sing = sg;
  }
  if (lane < (uint32_t)n) S.inlev[lane] = 0;
  if (lane + 32 < (uint32_t)n) S.inlev[lane + 32] = 0;
  __syncwarp();
  return starts;
}

// The search (sequential.cpp:216-670) for one graph.
struct W64Result {
  int32_t status;
  int num_aut;
  int64_t nodes;
};

// The root node (sequential.cpp:626-630): adjacency and the colour
// partition into shared memory, then the refinement with every cell active.
// The root's code is the first path's first code.
struct W64Root {
  uint64_t starts;
  int code;
  int32_t status;
};

static __device__ __noinline__ W64Root w64_root(const BatchArgs& A, int n, int64_t vo, int64_t eo,
                                                int64_t m, const int32_t* rp) {
  W64Smem& S = w64_smem();
  W64Root out{0ull, 0, kOk};
  const uint64_t starts = w64_load(n, rp, A.col + eo, A.color ? A.color + vo : nullptr, m);
  if (!starts) {
    out.status = kBadInput;
    return out;
  }
  const W64Refined r = w64_refine(n, starts, 0, starts);
  if (!r.ok) {
    out.status = kInternal;
    return out;
  }
  __syncwarp();
  if (lane_id() == 0) S.firstcode[0] = (uint16_t)r.code;
  __syncwarp();
  out.starts = r.starts;
  out.code = r.code;
  return out;
}

// The search below the root, with the root's partition in shared memory
// (`starts`, its refinement code `code`; level 1).
static __device__ __noinline__ W64Result w64_search_tree(const BatchArgs& A, int n, uint64_t starts,
                                                         int code, uint8_t* slot,
                                                         uint64_t deadline) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  uint8_t* reps = slot;
  uint8_t* auts = slot + (uint64_t)kW64Levels * 64u;
  W64Result res{kOk, 0, 1};
  const uint64_t full = low_mask((uint32_t)n);
  // Nauty_Sequential state (sequential.h:24-45), after the root node
  uint32_t level = 1, seqlen = 0, eqlevfirst = 0, first_seqlen = 0, best_seqlen = 0;
  int canon_level = 0, eqlevcanon = 0, comp_canon = 0, tcl = 0, num_aut = 0;
  bool first_found = false;
  int64_t nodes = 1;
  int32_t status = kOk;

  // the next refinement to run on the first path, given by its initially
  // active cells
  uint64_t pending = 0;
  uint64_t iter = 0;
  while (true) {
    if (pending) {
      const W64Refined r = w64_refine(n, starts, level, pending);
      pending = 0;
      if (!r.ok) {
        status = kInternal;
        break;
      }
      starts = r.starts;
      code = r.code;
      ++level;
      // the first path records its codes (sequential.cpp:254, 630)
      __syncwarp();
      if (lane == 0) S.firstcode[level - 1] = (uint16_t)code;
      __syncwarp();
      continue;
    }
    if (level == 0) break;
    if ((++iter & 63) == 0 && deadline &&
        __shfl_sync(GCL_FULL, lane == 0 ? global_ns() : 0ull, 0) > deadline) {
      status = kTimeout;
      break;
    }
    int bt = -1;       // backtrack target level
    int descend = -1;  // index of the target cell to branch from
    bool classify = false;
    const bool disc = starts == full;
    if (!first_found) {
      // first_path_node (sequential.cpp:216-257)
      if (disc) {
        // first_terminal (sequential.cpp:259-303)
        const Rows2 R = w64_leaf_rows(n);
        w64_store_leaf(n, R, S.first_cert, S.fpos);
        w64_store_leaf(n, R, S.best_cert, S.bpos);
        if (lane < seqlen) S.first_seq[lane] = S.best_seq[lane] = S.seq[lane];
        if (lane + 32 < seqlen) S.first_seq[lane + 32] = S.best_seq[lane + 32] = S.seq[lane + 32];
        if (lane < level) S.canoncode[lane] = S.firstcode[lane];
        if (lane + 32 < level) S.canoncode[lane + 32] = S.firstcode[lane + 32];
        __syncwarp();
        if (lane == 0) {
          S.firstcode[level] = (uint16_t)kSentinel;
          S.canoncode[level] = (uint16_t)kSentinel;
        }
        __syncwarp();
        eqlevfirst = level;
        first_seqlen = best_seqlen = seqlen;
        first_found = true;
        canon_level = eqlevcanon = (int)level;
        comp_canon = 0;
        bt = (int)level - 1;
      } else {
        if (tcl >= kW64Levels) {
          status = kInternal;
          break;
        }
        w64_select_tc(n, starts, tcl);
        ++tcl;
        descend = tcl - 1;
      }
    } else {
      // other_path_node (sequential.cpp:304-392)
      classify = true;
      if (!disc && (eqlevfirst == level || comp_canon >= 0)) {
        if (tcl < (int)level) {
          if (tcl >= kW64Levels) {
            status = kInternal;
            break;
          }
          w64_select_tc(n, starts, tcl);
          ++tcl;
        }
        const int idx = (int)level - 1;
        if (S.tc[idx].counter >= (uint32_t)n) {
          bt = (int)level - 1;
          classify = false;
        } else {
          if (num_aut > 0 && num_aut > S.tc[idx].last) {
            if (!w64_orbits(n, idx, num_aut, A.max_aut, seqlen, reps, auts,
                            reinterpret_cast<const uint64_t*>(auts + (uint64_t)A.aut_cap * 64u))) {
              status = kInternal;
              break;
            }
            __syncwarp();
            if (lane == 0) S.tc[idx].last = num_aut;
            __syncwarp();
          }
          descend = idx;
        }
      }
    }
    if (descend >= 0) {
      // next representative: smallest v >= counter with elems[v] == v
      const uint64_t r = S.tc[descend].repmask & ge_mask(S.tc[descend].counter);
      if (!r) {
        // the counter runs past the last vertex (sequential.cpp:359-365)
        __syncwarp();
        if (lane == 0) S.tc[descend].counter = (uint16_t)n;
        __syncwarp();
        bt = (int)level - 1;
        classify = false;
      } else {
        const uint32_t v = ctz64(r), t = S.tc[descend].first;
        __syncwarp();
        if (lane == 0) {
          S.tc[descend].counter = (uint16_t)(v + 1);
          S.seq[seqlen] = (uint8_t)v;
        }
        __syncwarp();
        ++seqlen;
        ++nodes;
        if (w64_individualize(n, level, v, t)) {
          starts |= bit64(t + 1);
          if (!first_found) {
            pending = bit64(t);  // refine and record firstcode
            continue;
          }
          const W64Refined rr = w64_refine(n, starts, level, bit64(t));
          if (!rr.ok) {
            status = kInternal;
            break;
          }
          starts = rr.starts;
          code = rr.code;
          ++level;
        } else if (!first_found) {
          __syncwarp();
          if (lane == 0) S.firstcode[level - 1] = (uint16_t)code;
          __syncwarp();
          continue;
        }
      }
    }
    if (classify) {
      // classify_node (sequential.cpp:396-624)
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
      Rows2 R{0ull, 0ull};
      if (eqlevfirst != Lv && comp_canon < 0) {
        dec = 4;
      } else if (starts == full) {
        R = w64_leaf_rows(n);
        if (eqlevfirst == Lv && w64_rows_equal(n, R, S.first_cert)) dec = 1;
        if (dec == 0) {
          if (comp_canon == 0) {
            if ((int)Lv < canon_level)
              comp_canon = 1;
            else
              comp_canon = w64_cmp_upper(n, R, S.best_cert);
          }
          dec = comp_canon == 0 ? 2 : (comp_canon > 0 ? 3 : 4);
        }
      }
      if (dec == 1 || dec == 2) {
        const uint32_t slot_i = (uint32_t)num_aut % A.max_aut;
        if (slot_i >= A.aut_cap) {
          status = kAutOverflow;
          break;
        }
        w64_store_aut(n, dec == 1 ? S.fpos : S.bpos,
                      slot_i < (uint32_t)kW64AutHead ? S.aut_head[slot_i]
                                                     : auts + (uint64_t)slot_i * 64u,
                      slot_i < (uint32_t)kW64AutHead
                          ? &S.fix_head[slot_i]
                          : reinterpret_cast<uint64_t*>(auts + (uint64_t)A.aut_cap * 64u) + slot_i);
        ++num_aut;
        const int g = dec == 1 ? w64_gca(S.first_seq, first_seqlen, seqlen)
                               : w64_gca(S.best_seq, best_seqlen, seqlen);
        bt = g >= 0 ? g : (int)Lv - 1;
      } else if (dec == 3) {
        canon_level = eqlevcanon = (int)Lv;
        comp_canon = 0;
        w64_store_leaf(n, R, S.best_cert, S.bpos);
        if (lane < seqlen) S.best_seq[lane] = S.seq[lane];
        if (lane + 32 < seqlen) S.best_seq[lane + 32] = S.seq[lane + 32];
        __syncwarp();
        if (lane == 0) S.canoncode[Lv] = (uint16_t)kSentinel;
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
      starts = w64_backtrack(n, starts, Lv);
      if (!starts) {
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
    }
  }
  res.status = status;
  res.num_aut = num_aut;
  res.nodes = nodes;
  return res;
}

__device__ __forceinline__ uint64_t w64_deadline(const BatchArgs& A) {
  if (!A.budget_ns) return 0;
  return __shfl_sync(GCL_FULL, lane_id() == 0 ? global_ns() : 0ull, 0) + A.budget_ns;
}

// The partition after the root refinement, handed from the warp that refined
// the root to the warp that searches below it: a header (starts, singleton
// vertices, code, graph id), then per vertex or position the adjacency mask, the cell
// member mask (at cell starts), the cell start, in_level and the singleton
// cell's vertex -- what the search reads of the root node.  Slots are whole
// 128-byte lines apart, so a warp never holds a line of a neighbouring slot
// in its L1 from before that slot was written.
__host__ __device__ constexpr uint64_t w64_root_slot_bytes() {
  return (32u + (uint64_t)kW64MaxN * (8u + 8u + 3u) + 127u) & ~127ull;
}

static __device__ __noinline__ void w64_save_root(uint8_t* dst, int g, int n, uint64_t starts,
                                                  int code) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  uint64_t* h = reinterpret_cast<uint64_t*>(dst);
  uint64_t* adj = h + 4;
  uint64_t* cm = adj + kW64MaxN;
  uint8_t* b = reinterpret_cast<uint8_t*>(cm + kW64MaxN);
  if (lane == 0) {
    h[0] = starts;
    h[1] = S.sing;
    h[2] = (uint64_t)(uint32_t)code;
    h[3] = (uint64_t)(uint32_t)g;
  }
  for (uint32_t v = lane; v < (uint32_t)n; v += 32) {
    adj[v] = S.adj[v];
    cm[v] = S.cmask[v];
    b[v] = S.cs[v];
    b[kW64MaxN + v] = S.inlev[v];
    b[2 * kW64MaxN + v] = S.pv[v];
  }
}

__device__ __forceinline__ int w64_root_graph(const uint8_t* src) {
  return (int)(uint32_t)reinterpret_cast<const uint64_t*>(src)[3];
}

// Search-cost class of a graph from its root partition: log2 of n times the
// vertices beyond one per cell (on the batched small-graph workload this
// estimate correlates 0.92 with nodes x n).  Graphs of class kW64InlineClass
// and above are searched at once by the warp that refined their root, so the
// longest searches of a batch start first.
constexpr int kW64CostClasses = 16;
constexpr int kW64InlineClass = 9;
__device__ __forceinline__ int w64_cost_class(int n, uint64_t starts) {
  const uint32_t est = (uint32_t)n * (uint32_t)(n - popc64(starts)) + 1u;
  return min(kW64CostClasses - 1, 31 - __clz((int)est));
}

static __device__ __noinline__ uint64_t w64_restore_root(const uint8_t* src, int n, int* code) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  const uint64_t* h = reinterpret_cast<const uint64_t*>(src);
  const uint64_t* adj = h + 4;
  const uint64_t* cm = adj + kW64MaxN;
  const uint8_t* b = reinterpret_cast<const uint8_t*>(cm + kW64MaxN);
  for (uint32_t v = lane; v < (uint32_t)n; v += 32) {
    S.adj[v] = adj[v];
    S.cmask[v] = cm[v];
    S.cs[v] = b[v];
    S.inlev[v] = b[kW64MaxN + v];
    S.pv[v] = b[2 * kW64MaxN + v];
  }
  const uint64_t starts = h[0];
  *code = (int)(uint32_t)h[2];
  if (lane == 0) {
    S.sing = h[1];
    S.firstcode[0] = (uint16_t)*code;
  }
  __syncwarp();
  return starts;
}

// The whole search of one graph: root node, then the tree below it.
static __device__ __forceinline__ W64Result w64_search(const BatchArgs& A, int n, int64_t vo,
                                                       int64_t eo, int64_t m, const int32_t* rp,
                                                       uint8_t* slot) {
  W64Result res{kOk, 0, 1};
  if (n == 0) return res;  // the reference visits the (discrete) root only
  const uint64_t deadline = w64_deadline(A);
  const W64Root root = w64_root(A, n, vo, eo, m, rp);
  if (root.status != kOk) {
    res.status = root.status;
    return res;
  }
  return w64_search_tree(A, n, root.starts, root.code, slot, deadline);
}

static __device__ __noinline__ void w64_write_outputs(const BatchArgs& A, int g, int n, int64_t vo) {
  W64Smem& S = w64_smem();
  const uint32_t lane = lane_id();
  if (A.out_label) {
    if (lane < (uint32_t)n) A.out_label[vo + S.bpos[lane]] = (int32_t)lane;
    if (lane + 32 < (uint32_t)n) A.out_label[vo + S.bpos[lane + 32]] = (int32_t)(lane + 32);
  }
  if (A.out_rows) {  // one word per row for n <= 64
    uint64_t* o = A.out_rows + A.roff[g];
    if (lane < (uint32_t)n) o[lane] = S.best_cert[lane];
    if (lane + 32 < (uint32_t)n) o[lane + 32] = S.best_cert[lane + 32];
  }
  if (A.out_dense) {
    uint8_t* o = A.out_dense + A.ooff[g];
    for (int r = 0; r < n; ++r) {
      const uint64_t row = S.best_cert[r];
      uint8_t* orow = o + (int64_t)r * n;
      if (lane < (uint32_t)n) orow[lane] = (uint8_t)((row >> lane) & 1ull);
      if (lane + 32 < (uint32_t)n) orow[lane + 32] = (uint8_t)((row >> (lane + 32)) & 1ull);
    }
  }
}

__device__ __forceinline__ void w64_canon_one(const BatchArgs& A, int g, uint8_t* slot) {
  const int64_t vo = A.voff[g];
  const int n = (int)(A.voff[g + 1] - vo);
  const int64_t eo = A.eoff[g];
  const W64Result r = w64_search(A, n, vo, eo, A.eoff[g + 1] - eo, A.rowptr + vo + g, slot);
  const uint32_t lane = lane_id();
  if (lane == 0) {
    A.status[g] = r.status;
    if (A.out_stats) {
      A.out_stats[2 * (int64_t)g] = r.num_aut;
      A.out_stats[2 * (int64_t)g + 1] = r.nodes;
    }
  }
  if (r.status == kOk) w64_write_outputs(A, g, n, vo);
  __syncwarp();
}

}  // namespace gcl
