/* canon_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * A plain-C restatement of the reference's sequential canonical labeler.
 * Every function names the reference file:line range whose behaviour it
 * restates.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load this file's library; the product never does.
 *
 * Parity pin: see canon_oracle.h.
 */
#include "canon_oracle.h"

#include <stdlib.h>
#include <string.h>

/* Invariant hash, partition_refinement.h:9-19 (nauty's MASH / CLEANUP). */
#define O_MASH(l, i) ((((l) ^ 065435u) + (i)) & 077777u)
#define O_CLEANUP(l) ((int)((l) % 077777u))
#define O_SENTINEL 077777

typedef struct {
  uint32_t first, length, in_level;
} ocell; /* CellStruct_s, structs.h:20-32 */

typedef struct {
  int32_t* elems; /* -1 = not in cell, else orbit representative */
  uint32_t first, length, counter;
  int last_num_aut;
} otc; /* TargetCell, structs.h:10-17 */

typedef struct {
  int n;
  const int32_t* rp;
  const int32_t* col;
  /* Partition_s, structs.h:65-86 */
  uint32_t* elem;
  ocell* lcs;
  uint32_t ncells;
  uint32_t level;
  uint32_t* seq;
  uint32_t seqlen;
  /* refinement scratch (partition_refinement.cpp:162-193) */
  uint8_t* active;
  uint32_t* deg;
  uint32_t* work;
  uint32_t* bucket;
} opart;

static int o_cell_index(const opart* P, uint32_t first) {
  /* cell_index_by_first, partition_refinement.cpp:12-25 */
  int lo = 0, hi = (int)P->ncells - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    uint32_t f = P->lcs[mid].first;
    if (first < f)
      hi = mid - 1;
    else if (first > f)
      lo = mid + 1;
    else
      return mid;
  }
  return -1;
}

static int o_discrete(const opart* P) {
  /* is_discrete, partition_refinement.cpp:70-78 */
  for (uint32_t i = 0; i < P->ncells; ++i)
    if (P->lcs[i].length != 1) return 0;
  return 1;
}

static const int32_t* o_color_key;
static int o_color_cmp(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  int cx = o_color_key ? o_color_key[x] : 0, cy = o_color_key ? o_color_key[y] : 0;
  if (cx != cy) return cx < cy ? -1 : 1;
  return x < y ? -1 : (x > y);
}

static void o_init_partition(opart* P, const int32_t* color) {
  /* initializePartition_s, partition_refinement.cpp:28-68: cells are colour
   * classes in ascending colour order, members by ascending id. */
  const int n = P->n;
  for (int v = 0; v < n; ++v) P->elem[v] = (uint32_t)v;
  o_color_key = color;
  qsort(P->elem, (size_t)n, sizeof(uint32_t), o_color_cmp);
  o_color_key = NULL;
  P->ncells = 0;
  P->level = 0;
  P->seqlen = 0;
  int s = 0;
  while (s < n) {
    int c = color ? color[P->elem[s]] : 0;
    int e = s + 1;
    while (e < n && (color ? color[P->elem[e]] : 0) == c) ++e;
    P->lcs[P->ncells].first = (uint32_t)s;
    P->lcs[P->ncells].length = (uint32_t)(e - s);
    P->lcs[P->ncells].in_level = 0;
    P->ncells++;
    s = e;
  }
}

/* Partition_s_refinement, partition_refinement.cpp:150-485.  `init` lists
 * the first positions of the initially active cells (NULL = all cells). */
static int o_refine(opart* P, const uint32_t* init, uint32_t ninit) {
  const uint32_t n = (uint32_t)P->n;
  uint8_t* active = P->active;
  uint32_t nactive = 0;
  memset(active, 0, n + 1);
#define ADD_ACT(f)                                  \
  do {                                              \
    uint32_t f_ = (f);                              \
    if (f_ < n && !active[f_]) active[f_] = 1, ++nactive; \
  } while (0)
#define DEL_ACT(f)                                  \
  do {                                              \
    uint32_t f_ = (f);                              \
    if (f_ < n && active[f_]) active[f_] = 0, --nactive; \
  } while (0)
  if (!init) {
    for (uint32_t i = 0; i < P->ncells; ++i) ADD_ACT(P->lcs[i].first);
  } else {
    for (uint32_t i = 0; i < ninit; ++i) ADD_ACT(init[i]);
  }
  uint64_t lc = (uint64_t)P->ncells;
  uint32_t* deg = P->deg;
  uint32_t* bucket = P->bucket;
  memset(deg, 0, n * sizeof(uint32_t));
  int hint = 0;

  while (!o_discrete(P) && nactive > 0) {
    /* splitter: hint if active, else next active after it, else wrap
     * (partition_refinement.cpp:202-226) */
    int s1 = -1;
    if (hint >= 0 && (uint32_t)hint < n && active[hint]) {
      s1 = hint;
    } else {
      for (uint32_t p = (uint32_t)hint + 1; p < n; ++p)
        if (active[p]) { s1 = (int)p; break; }
      if (s1 < 0)
        for (uint32_t p = 0; p < n; ++p)
          if (active[p]) { s1 = (int)p; break; }
    }
    uint32_t split1 = (uint32_t)s1;
    DEL_ACT(split1);
    ocell spl = P->lcs[o_cell_index(P, split1)];
    uint32_t split2 = split1 + spl.length - 1;
    lc = O_MASH(lc, (uint64_t)(uint32_t)(split1 + split2));
    if (spl.length > 1) lc = O_MASH(lc, (uint64_t)spl.length);

    /* neighbour counts into the splitter (:244-251) */
    for (uint32_t i = 0; i < spl.length; ++i) {
      uint32_t w = P->elem[spl.first + i];
      for (int32_t e = P->rp[w]; e < P->rp[w + 1]; ++e) ++deg[P->col[e]];
    }

    for (int ci = 0; ci < (int)P->ncells; ++ci) {
      ocell cell = P->lcs[ci];
      if (cell.length == 1) continue;
      uint32_t* cv = &P->elem[cell.first];
      uint32_t common = deg[cv[0]], bmin = common, bmax = common;
      int is_common = 1;
      for (uint32_t j = 1; j < cell.length; ++j) {
        uint32_t d = deg[cv[j]];
        if (d != common) is_common = 0;
        if (d < bmin) bmin = d;
        if (d > bmax) bmax = d;
      }
      if (is_common) {
        if (spl.length > 1) lc = O_MASH(lc, (uint64_t)(uint32_t)(common + cell.first));
        continue;
      }
      for (uint32_t d = bmin; d <= bmax; ++d) bucket[d] = 0;
      for (uint32_t j = 0; j < cell.length; ++j) ++bucket[deg[cv[j]]];
      uint32_t nnew = 0;
      if (spl.length == 1) {
        if (bmin <= 1 && bmax >= 1 && bucket[1] > 0) ++nnew;
        if (bmin == 0 && bucket[0] > 0) ++nnew;
      } else {
        for (uint32_t d = bmin; d <= bmax; ++d)
          if (bucket[d]) ++nnew;
      }
      if (nnew > 1)
        for (int j = (int)P->ncells - 1; j > ci; --j) P->lcs[j + (int)nnew - 1] = P->lcs[j];

      /* fragment descriptors, ascending count ([1, 0] for a singleton
       * splitter) (:326-373) */
      uint32_t fidx = 0, first = cell.first, maxsz = 0, maxidx = 0;
      uint32_t order[2] = {1, 0};
      uint32_t nd = spl.length == 1 ? 2 : bmax - bmin + 1;
      for (uint32_t k = 0; k < nd; ++k) {
        uint32_t dv;
        if (spl.length == 1) {
          dv = order[k];
          if (!(bmin <= dv && bmax >= dv)) continue;
        } else {
          dv = bmin + k;
        }
        uint32_t size = bucket[dv];
        if (!size) continue;
        ocell* nc = &P->lcs[ci + (int)fidx];
        nc->first = first;
        nc->length = size;
        nc->in_level = P->level + 1;
        if (spl.length > 1) lc = O_MASH(lc, (uint64_t)(uint32_t)(dv + nc->first));
        if (size > maxsz) maxsz = size, maxidx = fidx;
        bucket[dv] = first - cell.first;
        first += size;
        ++fidx;
      }
      P->ncells += nnew - 1;
      /* stable reorder inside each fragment (:381-391) */
      for (uint32_t j = 0; j < cell.length; ++j) {
        uint32_t v = cv[j];
        P->work[bucket[deg[v]]++] = v;
      }
      memcpy(cv, P->work, cell.length * sizeof(uint32_t));

      int was_active = active[cell.first] != 0;
      if (spl.length == 1) {
        /* (:399-409) */
        uint32_t nb = P->lcs[ci].length;
        uint32_t nn = nnew > 1 ? P->lcs[ci + 1].length : 0;
        if (nb > 0 && nn > 0) lc = O_MASH(lc, (uint64_t)(uint32_t)(cell.first + nb - 1));
        /* active set (:414-435) */
        if (was_active || nb >= nn) {
          if (nnew > 1) {
            uint32_t fs = P->lcs[ci + 1].first;
            ADD_ACT(fs);
            if (P->lcs[ci + 1].length == 1) hint = (int)fs;
          }
        } else {
          uint32_t fs = P->lcs[ci].first;
          ADD_ACT(fs);
          if (P->lcs[ci].length == 1) hint = (int)fs;
        }
      } else {
        /* (:436-460) */
        for (uint32_t f = 0; f < nnew; ++f) {
          ocell* fr = &P->lcs[ci + (int)f];
          if (fr->first != cell.first) {
            ADD_ACT(fr->first);
            if (fr->length == 1) hint = (int)fr->first;
          }
        }
        if (!was_active) {
          ADD_ACT(cell.first);
          DEL_ACT(P->lcs[ci + (int)maxidx].first);
        }
      }
      /* the last fragment inherits the old in_level (:463-465) */
      if (cell.in_level != P->level + 1 && nnew > 0)
        P->lcs[ci + (int)nnew - 1].in_level = cell.in_level;
      ci = ci + (int)nnew - 1;
    }
    memset(deg, 0, n * sizeof(uint32_t));
  }
#undef ADD_ACT
#undef DEL_ACT
  lc = O_MASH(lc, (uint64_t)P->ncells);
  P->level++;
  return O_CLEANUP(lc);
}

/* split_by_and_refine, partition_refinement.cpp:486-539 */
static void o_individualize(opart* P, uint32_t vertex, int* code, uint32_t tc_first) {
  int ci = o_cell_index(P, tc_first);
  ocell cell = P->lcs[ci];
  if (cell.length == 1) return;
  uint32_t s = cell.first, e = cell.first + cell.length, vi = s;
  while (vi < e && P->elem[vi] != vertex) ++vi;
  if (vi > s) {
    for (uint32_t i = vi; i > s; --i) P->elem[i] = P->elem[i - 1];
    P->elem[s] = vertex;
  }
  ocell rest = {cell.first + 1, cell.length - 1, cell.in_level};
  for (int i = (int)P->ncells - 1; i > ci; --i) P->lcs[i + 1] = P->lcs[i];
  P->lcs[ci + 1] = rest;
  P->ncells++;
  cell.length = 1;
  cell.in_level = P->level + 1;
  P->lcs[ci] = cell;
  uint32_t act = cell.first;
  *code = o_refine(P, &act, 1);
}

static int o_u32_cmp(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return x < y ? -1 : (x > y);
}

/* reconstruct_at_level, partition_refinement.cpp:541-604 */
static void o_reconstruct(opart* P, uint32_t L, uint32_t* eqlev_first, int* eqlev_canon,
                          int* comp_canon) {
  if (L < 1) return;
  for (uint32_t i = 0; i < P->ncells;) {
    if (P->lcs[i].in_level <= L) {
      ++i;
      continue;
    }
    uint32_t first = P->lcs[i].first, j = i + 1, len = P->lcs[i].length;
    while (j < P->ncells && P->lcs[j].in_level > L) len += P->lcs[j++].length;
    if (j < P->ncells) len += P->lcs[j].length;
    qsort(P->elem + first, len, sizeof(uint32_t), o_u32_cmp);
    P->lcs[i].first = first;
    P->lcs[i].length = len;
    P->lcs[i].in_level = P->lcs[j].in_level;
    uint32_t drop = j - i;
    if (drop > 0) {
      for (uint32_t k = j + 1; k < P->ncells; ++k) P->lcs[k - drop] = P->lcs[k];
      P->ncells -= drop;
    }
    ++i;
  }
  if (L < *eqlev_first) *eqlev_first = L;
  if ((int)L <= *eqlev_canon) {
    *eqlev_canon = (int)L;
    *comp_canon = 0;
  }
  P->level = L;
}

/* ------------------------------------------------------------------------ */
/* Search state: class Nauty_Sequential, sequential.h:12-71                   */

typedef struct {
  opart P;
  int n;
  unsigned max_aut;
  uint32_t* auts; /* ring of max_aut perms (sequential.cpp:515, 552) */
  int num_aut;
  int64_t nodes;
  int code;
  int canon_level, eqlevcanon, comp_canon;
  uint32_t eqlevfirst;
  int* canon_code;
  int* firstcode;
  otc* tcs;
  int tc_level_reached;
  /* Leaf_s, structs.h:34-61 */
  uint32_t *first_seq, *best_seq;
  uint32_t first_seqlen, best_seqlen;
  uint32_t *first_label, *best_label;
  uint8_t *best_hash, *cur_hash;
  int first_discovered;
  /* scratch */
  uint32_t *perm, *aut, *dsu;
  int* subgroup;
} osearch;

/* buildPermutedFlatAdjacencyMatrixArray(discrete_partition_to_perm(P)),
 * CSRGraph.cpp:332-351 and perm_group.cpp:118-127 */
static void o_leaf_matrix(osearch* S, uint8_t* out) {
  const int n = S->n;
  for (int i = 0; i < n; ++i) S->perm[S->P.elem[i]] = (uint32_t)i;
  memset(out, 0, (size_t)n * (size_t)n);
  for (int i = 0; i < n; ++i) {
    uint32_t pi = S->perm[i];
    for (int32_t k = S->P.rp[i]; k < S->P.rp[i + 1]; ++k) {
      uint32_t pj = S->perm[S->P.col[k]];
      out[(size_t)pi * n + pj] = 1;
      out[(size_t)pj * n + pi] = 1;
    }
  }
}

/* compare_adj_upper, sequential.cpp:114-124 */
static int o_cmp_upper(const uint8_t* A, const uint8_t* B, int n) {
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      uint8_t a = A[(size_t)i * n + j], b = B[(size_t)i * n + j];
      if (a != b) return a ? 1 : -1;
    }
  return 0;
}

static int o_has_edge(const opart* P, uint32_t u, uint32_t v) {
  int32_t lo = P->rp[u], hi = P->rp[u + 1] - 1;
  while (lo <= hi) {
    int32_t mid = (lo + hi) >> 1;
    uint32_t c = (uint32_t)P->col[mid];
    if (c == v) return 1;
    if (c < v)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  return 0;
}

/* isAutomorphism, sequential.cpp:127-167.  The reference checks all n^2
 * pairs; for a bijection that is equivalent to "equal degrees and every
 * edge maps to an edge", which is what is checked here (same boolean). */
static int o_is_aut(const osearch* S, const uint32_t* perm) {
  const opart* P = &S->P;
  for (int u = 0; u < S->n; ++u) {
    uint32_t pu = perm[u];
    if (P->rp[u + 1] - P->rp[u] != P->rp[pu + 1] - P->rp[pu]) return 0;
  }
  for (int u = 0; u < S->n; ++u)
    for (int32_t k = P->rp[u]; k < P->rp[u + 1]; ++k)
      if (!o_has_edge(P, perm[u], perm[P->col[k]])) return 0;
  return 1;
}

/* get_gca_level, sequential.cpp:183-213 */
static int o_gca(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb) {
  uint32_t m = na < nb ? na : nb;
  for (uint32_t i = 0; i < m; ++i)
    if (a[i] != b[i]) return (int)i + 1;
  return -1;
}

/* target_cell_selector with hint -1, partition_refinement.cpp:607-655 */
static int o_select_tc(osearch* S) {
  opart* P = &S->P;
  int tc = -1;
  for (uint32_t i = 0; i < P->ncells; ++i)
    if (P->lcs[i].length > 1) { tc = (int)i; break; }
  if (tc >= 0) {
    otc* t = &S->tcs[S->tc_level_reached];
    for (int v = 0; v < S->n; ++v) t->elems[v] = -1;
    ocell c = P->lcs[tc];
    for (uint32_t k = 0; k < c.length; ++k) {
      int v = (int)P->elem[c.first + k];
      t->elems[v] = v;
    }
    t->length = c.length;
    t->counter = 0;
    t->last_num_aut = 0;
    t->first = c.first;
    S->tc_level_reached++;
  }
  return tc;
}

/* subgroup_fixing_sequence + compute_orbits_fast, perm_group.cpp:5-116 */
static void o_orbits(osearch* S, otc* t) {
  const int n = S->n;
  int limit = S->num_aut < (int)S->max_aut ? S->num_aut : (int)S->max_aut;
  int from = t->last_num_aut == -1 ? 0 : t->last_num_aut;
  int nsub = 0;
  for (int i = from; i < limit; ++i) {
    const uint32_t* pm = &S->auts[(size_t)i * n];
    int fixes = 1;
    for (uint32_t j = 0; j < S->P.seqlen; ++j)
      if (pm[S->P.seq[j]] != S->P.seq[j]) { fixes = 0; break; }
    if (fixes) S->subgroup[nsub++] = i;
  }
  if (nsub == 0) return;
  uint32_t* par = S->dsu;
  for (int v = 0; v < n; ++v) par[v] = t->elems[v] != -1 ? (uint32_t)t->elems[v] : (uint32_t)v;
  for (int s = 0; s < nsub; ++s) {
    const uint32_t* pm = &S->auts[(size_t)S->subgroup[s] * n];
    for (int v = 0; v < n; ++v) {
      uint32_t img = pm[v];
      if ((uint32_t)v == img) continue;
      uint32_t a = (uint32_t)v, b = img;
      while (par[a] != a) a = par[a];
      while (par[b] != b) b = par[b];
      if (a == b) continue;
      if (a < b)
        par[b] = a;
      else
        par[a] = b;
    }
  }
  for (int v = 0; v < n; ++v)
    if (t->elems[v] != -1) {
      uint32_t a = (uint32_t)v;
      while (par[a] != a) a = par[a];
      t->elems[v] = (int32_t)a;
    }
}

/* backtrack_to, sequential.cpp:650-670 */
static void o_backtrack(osearch* S, uint32_t L) {
  if (L == 0) {
    S->P.level = 0;
    return;
  }
  o_reconstruct(&S->P, L, &S->eqlevfirst, &S->eqlevcanon, &S->comp_canon);
  S->P.seqlen = L - 1;
  S->tc_level_reached = (int)L;
  S->P.level = L;
}

static int o_next_rep(osearch* S, otc* t) {
  while (t->counter < (uint32_t)S->n && t->elems[t->counter] != (int32_t)t->counter) ++t->counter;
  return t->counter < (uint32_t)S->n;
}

/* first_terminal, sequential.cpp:259-303 */
static void o_first_terminal(osearch* S) {
  opart* P = &S->P;
  S->eqlevfirst = P->level;
  S->firstcode[P->level] = O_SENTINEL;
  o_leaf_matrix(S, S->best_hash);
  S->first_seqlen = S->best_seqlen = P->seqlen;
  for (uint32_t i = 0; i < P->seqlen; ++i) S->first_seq[i] = S->best_seq[i] = P->seq[i];
  for (int j = 0; j < S->n; ++j) S->first_label[j] = S->best_label[j] = P->elem[j];
  S->first_discovered = 1;
  S->canon_level = S->eqlevcanon = (int)P->level;
  S->comp_canon = 0;
  for (uint32_t i = 0; i < P->level; ++i) S->canon_code[i] = S->firstcode[i];
  S->canon_code[P->level] = O_SENTINEL;
}

/* first_path_node, sequential.cpp:216-257 */
static void o_first_path_node(osearch* S) {
  opart* P = &S->P;
  if (o_discrete(P)) {
    o_first_terminal(S);
    o_backtrack(S, P->level - 1);
    return;
  }
  o_select_tc(S);
  otc* t = &S->tcs[S->tc_level_reached - 1];
  o_next_rep(S, t);
  uint32_t v = t->counter++;
  ++S->nodes;
  P->seq[P->seqlen++] = v;
  o_individualize(P, v, &S->code, t->first);
  S->firstcode[P->level - 1] = S->code;
}

static void o_store_aut(osearch* S, const uint32_t* label) {
  const int n = S->n;
  for (int j = 0; j < n; ++j) S->aut[label[j]] = S->P.elem[j];
  unsigned idx = (unsigned)S->num_aut % S->max_aut;
  memcpy(&S->auts[(size_t)idx * n], S->aut, (size_t)n * sizeof(uint32_t));
  S->num_aut++;
}

/* classify_node, sequential.cpp:396-624 */
static void o_classify(osearch* S) {
  opart* P = &S->P;
  const int n = S->n;
  const int L = (int)P->level;
  if (S->eqlevfirst == (uint32_t)(L - 1) && S->code == S->firstcode[L - 1]) S->eqlevfirst = (uint32_t)L;
  if (S->eqlevcanon == L - 1) {
    if (S->code < S->canon_code[L - 1])
      S->comp_canon = -1;
    else if (S->code > S->canon_code[L - 1])
      S->comp_canon = 1;
    else {
      S->comp_canon = 0;
      S->eqlevcanon = L;
    }
  }
  if (S->comp_canon > 0) S->canon_code[L - 1] = S->code;

  int dec = 0;
  if (S->eqlevfirst != (uint32_t)L && S->comp_canon < 0) {
    dec = 4;
  } else if (o_discrete(P)) {
    if (S->eqlevfirst == (uint32_t)L) {
      for (int j = 0; j < n; ++j) S->aut[S->first_label[j]] = P->elem[j];
      if (o_is_aut(S, S->aut)) dec = 1;
    }
    if (dec == 0) {
      if (S->comp_canon == 0) {
        if (L < S->canon_level) {
          S->comp_canon = 1;
        } else {
          o_leaf_matrix(S, S->cur_hash);
          S->comp_canon = o_cmp_upper(S->cur_hash, S->best_hash, n);
        }
      }
      dec = S->comp_canon == 0 ? 2 : (S->comp_canon > 0 ? 3 : 4);
    }
  }

  switch (dec) {
    case 1: {
      o_store_aut(S, S->first_label);
      int g = o_gca(S->first_seq, S->first_seqlen, P->seq, P->seqlen);
      o_backtrack(S, g >= 0 ? (uint32_t)g : (uint32_t)(L - 1));
      break;
    }
    case 2: {
      o_store_aut(S, S->best_label);
      int g = o_gca(S->best_seq, S->best_seqlen, P->seq, P->seqlen);
      o_backtrack(S, g >= 0 ? (uint32_t)g : (uint32_t)(L - 1));
      break;
    }
    case 3: {
      S->canon_level = S->eqlevcanon = L;
      S->comp_canon = 0;
      S->canon_code[L] = O_SENTINEL;
      for (int j = 0; j < n; ++j) S->best_label[j] = P->elem[j];
      o_leaf_matrix(S, S->best_hash);
      for (uint32_t i = 0; i < P->seqlen; ++i) S->best_seq[i] = P->seq[i];
      S->best_seqlen = P->seqlen;
      o_backtrack(S, (uint32_t)(L - 1));
      break;
    }
    case 4:
      o_backtrack(S, (uint32_t)(L - 1));
      break;
    default:
      break;
  }
}

/* other_path_node, sequential.cpp:304-392 */
static void o_other_path_node(osearch* S) {
  opart* P = &S->P;
  if (!o_discrete(P) && (S->eqlevfirst == P->level || S->comp_canon >= 0)) {
    if (S->tc_level_reached < (int)P->level) o_select_tc(S);
    otc* t = &S->tcs[P->level - 1];
    if (t->counter >= (uint32_t)S->n) {
      o_backtrack(S, P->level - 1);
      return;
    }
    if (S->num_aut > 0 && S->num_aut > t->last_num_aut) {
      o_orbits(S, t);
      t->last_num_aut = S->num_aut;
    }
    if (!o_next_rep(S, t)) {
      o_backtrack(S, P->level - 1);
      return;
    }
    uint32_t v = t->counter++;
    ++S->nodes;
    P->seq[P->seqlen++] = v;
    o_individualize(P, v, &S->code, t->first);
  }
  o_classify(S);
}

static void o_free(osearch* S) {
  opart* P = &S->P;
  free(P->elem);
  free(P->lcs);
  free(P->seq);
  free(P->active);
  free(P->deg);
  free(P->work);
  free(P->bucket);
  free(S->auts);
  free(S->canon_code);
  free(S->firstcode);
  if (S->tcs) {
    for (int i = 0; i <= S->n; ++i) free(S->tcs[i].elems);
    free(S->tcs);
  }
  free(S->first_seq);
  free(S->best_seq);
  free(S->first_label);
  free(S->best_label);
  free(S->best_hash);
  free(S->cur_hash);
  free(S->perm);
  free(S->aut);
  free(S->dsu);
  free(S->subgroup);
}

static int o_alloc(osearch* S, int n, unsigned max_aut) {
  size_t N = (size_t)(n > 0 ? n : 1);
  opart* P = &S->P;
  P->elem = malloc(N * 4);
  P->lcs = malloc((N + 1) * sizeof(ocell));
  P->seq = malloc(N * 4);
  P->active = malloc(N + 1);
  P->deg = malloc(N * 4);
  P->work = malloc(N * 4);
  P->bucket = malloc((N + 1) * 4);
  S->auts = malloc((size_t)max_aut * N * 4);
  S->canon_code = malloc((N + 2) * sizeof(int));
  S->firstcode = malloc((N + 2) * sizeof(int));
  S->tcs = calloc(N + 1, sizeof(otc));
  S->first_seq = malloc(N * 4);
  S->best_seq = malloc(N * 4);
  S->first_label = malloc(N * 4);
  S->best_label = malloc(N * 4);
  S->best_hash = malloc(N * N);
  S->cur_hash = malloc(N * N);
  S->perm = malloc(N * 4);
  S->aut = malloc(N * 4);
  S->dsu = malloc(N * 4);
  S->subgroup = malloc((size_t)max_aut * sizeof(int));
  if (!P->elem || !P->lcs || !P->seq || !P->active || !P->deg || !P->work || !P->bucket ||
      !S->auts || !S->canon_code || !S->firstcode || !S->tcs || !S->first_seq ||
      !S->best_seq || !S->first_label || !S->best_label || !S->best_hash || !S->cur_hash ||
      !S->perm || !S->aut || !S->dsu || !S->subgroup)
    return -1;
  for (size_t i = 0; i <= N; ++i) {
    S->tcs[i].elems = malloc(N * 4);
    if (!S->tcs[i].elems) return -1;
  }
  return 0;
}

int gcl_oracle_canon(int n, const int32_t* rowptr, const int32_t* col, const int32_t* color,
                     unsigned max_aut, uint8_t* out_nxn, int32_t* label_out,
                     gcl_oracle_stats* st) {
  if (n < 0 || max_aut == 0 || !rowptr || (n > 0 && rowptr[n] > 0 && !col)) return -1;
  osearch S;
  memset(&S, 0, sizeof S);
  S.n = n;
  S.max_aut = max_aut;
  if (o_alloc(&S, n, max_aut)) {
    S.n = n > 0 ? n : 1;
    o_free(&S);
    return -1;
  }
  opart* P = &S.P;
  P->n = n;
  P->rp = rowptr;
  P->col = col;
  o_init_partition(P, color);

  /* search_tree_traversal, sequential.cpp:626-648 */
  S.code = o_refine(P, NULL, 0);
  S.firstcode[P->level - 1] = S.code;
  S.nodes = 1;
  while (P->level >= 1) {
    if (!S.first_discovered)
      o_first_path_node(&S);
    else
      o_other_path_node(&S);
  }
  if (out_nxn) memcpy(out_nxn, S.best_hash, (size_t)n * (size_t)n);
  if (label_out)
    for (int i = 0; i < n; ++i) label_out[i] = (int32_t)S.best_label[i];
  if (st) {
    st->num_aut = S.num_aut;
    st->nodes = S.nodes;
  }
  o_free(&S);
  return 0;
}

int gcl_oracle_canon_batch(int count, const int64_t* voff, const int64_t* eoff,
                           const int32_t* rowptr_arena, const int32_t* col_arena,
                           const int32_t* color_arena, unsigned max_aut, uint8_t* out_arena,
                           const int64_t* ooff, int32_t* label_arena, gcl_oracle_stats* stats) {
  for (int g = 0; g < count; ++g) {
    int n = (int)(voff[g + 1] - voff[g]);
    int rc = gcl_oracle_canon(n, rowptr_arena + voff[g] + g, col_arena + eoff[g],
                              color_arena ? color_arena + voff[g] : NULL, max_aut,
                              out_arena ? out_arena + ooff[g] : NULL,
                              label_arena ? label_arena + voff[g] : NULL,
                              stats ? stats + g : NULL);
    if (rc) return rc;
  }
  return 0;
}

int gcl_oracle_root_refine(int n, const int32_t* rowptr, const int32_t* col, const int32_t* color,
                           int32_t* elem_out, int32_t* cell_start_out) {
  if (n <= 0) return -1;
  opart P;
  memset(&P, 0, sizeof P);
  size_t N = (size_t)n;
  P.n = n;
  P.rp = rowptr;
  P.col = col;
  P.elem = malloc(N * 4);
  P.lcs = malloc((N + 1) * sizeof(ocell));
  P.seq = malloc(N * 4);
  P.active = malloc(N + 1);
  P.deg = malloc(N * 4);
  P.work = malloc(N * 4);
  P.bucket = malloc((N + 1) * 4);
  int code = -1;
  if (P.elem && P.lcs && P.seq && P.active && P.deg && P.work && P.bucket) {
    o_init_partition(&P, color);
    code = o_refine(&P, NULL, 0);
    for (int i = 0; i < n; ++i) elem_out[i] = (int32_t)P.elem[i];
    for (uint32_t c = 0; c < P.ncells; ++c)
      for (uint32_t k = 0; k < P.lcs[c].length; ++k)
        cell_start_out[P.lcs[c].first + k] = (int32_t)P.lcs[c].first;
  }
  free(P.elem);
  free(P.lcs);
  free(P.seq);
  free(P.active);
  free(P.deg);
  free(P.work);
  free(P.bucket);
  return code;
}
