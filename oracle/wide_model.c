/* wide_model.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU model of the GPU's wide search (many workers on one search tree,
 * csrc/canon_wide.cuh) built on the C restatement of the reference's
 * sequential search (canon_oracle.c, included below for its internal
 * functions).  W simulated workers take the first path's siblings as work
 * items, deepest level first, and step through the reference's DFS one node
 * at a time, in round-robin or seeded random order; they share an
 * append-only automorphism store and a best leaf, and each keeps a private
 * copy of the best leaf.  The two rules the wide search changes are the ones
 * modelled:
 *   - a leaf equivalent to a best leaf found outside the current item only
 *     records the automorphism and steps back one level;
 *   - a node worse than the private best (after adopting a newer shared best)
 *     and off the first path's trail is pruned at once.
 * tests/test_wide_model.py checks that every schedule gives the sequential
 * canonical matrix, and that the sequential result is the maximum over all
 * leaves (exhaustive search) -- the property the wide search rests on.
 * With `donate` set, a busy worker hands its shallowest untried child to an
 * idle worker (work sharing below the first path's siblings).
 * With `gate` set, an item starts only once every item of the deeper levels
 * is done, as the GPU's level gate orders them; gate | 8 adds the probe:
 * the first item of each level runs alone, the rest of the level once it is
 * done or 2D rounds after it started, whichever comes first (the GPU waits
 * twice the first path's duration; GCL_OPT_WIDE_PROBE); `rounds` counts the
 * scheduling rounds (every worker takes one step per round), the model's
 * measure of the search's parallel time; rounds[1] and rounds[2] receive the
 * first leaf's level D and the number of items.
 *
 * Built with the oracle (oracle/Makefile) into libgcl_wide_model.so; only
 * tests load it.
 */
#include "canon_oracle.c"

#include <stdio.h>

typedef struct {
  int n;
  uint32_t D; /* level of the first leaf */
  int* firstcode;
  uint32_t* first_seq;
  uint32_t first_seqlen;
  uint32_t* first_label;
  opart leafP;
  uint32_t* item_k;
  uint32_t* item_v;
  int nitems, next_item;
  int* g_code; /* shared best leaf */
  int g_level;
  uint32_t* g_label;
  uint32_t* g_seq;
  uint32_t g_seqlen;
  uint8_t* g_hash;
  int g_version;
  uint32_t* auts; /* append-only store */
  int naut, cap;
  long nodes;
  /* how often the changed rules fired: [0] a leaf equivalent to a best found
   * outside the item, [1] a node pruned as worse than the private best,
   * [2] a leaf that beat the private best but not a newer shared one */
  long events[4]; /* [3]: handed-over subtrees whose replayed codes differed */
  int replay;     /* receivers rebuild a handed-over parent from the first leaf */
} wm_shared;

typedef struct {
  osearch S;
  int* pathcode; /* pathcode[L-1] = code of the node at level L on the path */
  int busy;
  uint32_t item_k;
  int best_local; /* the private best was found in this item (or is the first leaf) */
  int version;
  int gift;       /* the current work is a donated subtree, not a first-path item */
} wm_worker;

/* A subtree handed over by a busy worker: the parent node (its partition at
 * level L, its L-1 individualized vertices and L codes) and the child v. */
typedef struct {
  opart P;
  uint32_t L;
  uint32_t* seq;
  int* pathcode;
  uint32_t v;
} wm_gift;

static void wm_copy_part(opart* d, const opart* s, int n) {
  memcpy(d->elem, s->elem, (size_t)n * 4);
  memcpy(d->lcs, s->lcs, ((size_t)n + 1) * sizeof(ocell));
  d->ncells = s->ncells;
  d->level = s->level;
}

/* comparison state of the path of level Lp against the private best */
static void wm_recompare(wm_worker* w, uint32_t Lp) {
  osearch* S = &w->S;
  uint32_t i = 0;
  while (i < Lp && (int)i < S->canon_level && w->pathcode[i] == S->canon_code[i]) ++i;
  if (i == Lp) {
    S->eqlevcanon = (int)Lp;
    S->comp_canon = 0;
    return;
  }
  S->eqlevcanon = (int)i;
  int bc = (int)i < S->canon_level ? S->canon_code[i] : O_SENTINEL;
  S->comp_canon = w->pathcode[i] < bc ? -1 : 1;
  if (S->comp_canon > 0)
    for (uint32_t j = i; j < Lp; ++j) S->canon_code[j] = w->pathcode[j];
}

static void wm_adopt(wm_worker* w, wm_shared* G) {
  osearch* S = &w->S;
  int n = G->n;
  for (int i = 0; i < G->g_level; ++i) S->canon_code[i] = G->g_code[i];
  S->canon_code[G->g_level] = O_SENTINEL;
  S->canon_level = G->g_level;
  memcpy(S->best_label, G->g_label, (size_t)n * 4);
  memcpy(S->best_seq, G->g_seq, (size_t)G->g_seqlen * 4);
  S->best_seqlen = G->g_seqlen;
  memcpy(S->best_hash, G->g_hash, (size_t)n * n);
  w->version = G->g_version;
}

static void wm_store_aut(wm_shared* G, osearch* S, const uint32_t* label) {
  int n = G->n;
  for (int j = 0; j < n; ++j) S->aut[label[j]] = S->P.elem[j];
  if (G->naut < G->cap) {
    memcpy(&G->auts[(size_t)G->naut * n], S->aut, (size_t)n * 4);
    G->naut++;
  }
}

static void wm_sync_auts(wm_worker* w, wm_shared* G) {
  w->S.auts = G->auts;
  w->S.num_aut = G->naut;
  w->S.max_aut = (unsigned)G->cap;
}

/* a leaf better than the private best: 1 if it became the shared best */
static int wm_publish(wm_worker* w, wm_shared* G, uint32_t L) {
  osearch* S = &w->S;
  int n = G->n, cmp = 0;
  for (uint32_t i = 0; i < L && (int)i < G->g_level; ++i)
    if (w->pathcode[i] != G->g_code[i]) {
      cmp = w->pathcode[i] < G->g_code[i] ? -1 : 1;
      break;
    }
  if (cmp == 0) {
    if ((int)L < G->g_level)
      cmp = 1;
    else if ((int)L > G->g_level)
      cmp = -1;
    else
      cmp = o_cmp_upper(S->cur_hash, G->g_hash, n);
  }
  if (cmp > 0) {
    for (uint32_t j = 0; j < L; ++j) G->g_code[j] = w->pathcode[j];
    G->g_level = (int)L;
    memcpy(G->g_label, S->P.elem, (size_t)n * 4);
    memcpy(G->g_seq, S->P.seq, (size_t)S->P.seqlen * 4);
    G->g_seqlen = S->P.seqlen;
    memcpy(G->g_hash, S->cur_hash, (size_t)n * n);
    G->g_version++;
    return 1;
  }
  if (cmp == 0) wm_store_aut(G, S, G->g_label); /* equivalent to the shared best */
  return 0;
}

/* classify_node (sequential.cpp:396-624) with the wide-search rules */
static void wm_classify(wm_worker* w, wm_shared* G) {
  osearch* S = &w->S;
  opart* P = &S->P;
  const int n = S->n;
  const int L = (int)P->level;
  w->pathcode[L - 1] = S->code;
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
  wm_sync_auts(w, G);
  switch (dec) {
    case 1: {
      wm_store_aut(G, S, S->first_label);
      int g = o_gca(S->first_seq, S->first_seqlen, P->seq, P->seqlen);
      o_backtrack(S, g >= 0 ? (uint32_t)g : (uint32_t)(L - 1));
      break;
    }
    case 2: {
      wm_store_aut(G, S, S->best_label);
      if (!w->best_local) G->events[0]++;
      int g = w->best_local ? o_gca(S->best_seq, S->best_seqlen, P->seq, P->seqlen) : -1;
      o_backtrack(S, g >= 0 ? (uint32_t)g : (uint32_t)(L - 1));
      break;
    }
    case 3:
      o_leaf_matrix(S, S->cur_hash);
      if (wm_publish(w, G, (uint32_t)L)) {
        S->canon_level = S->eqlevcanon = L;
        S->comp_canon = 0;
        for (int j = 0; j < L; ++j) S->canon_code[j] = w->pathcode[j];
        S->canon_code[L] = O_SENTINEL;
        memcpy(S->best_label, P->elem, (size_t)n * 4);
        memcpy(S->best_hash, S->cur_hash, (size_t)n * n);
        memcpy(S->best_seq, P->seq, (size_t)P->seqlen * 4);
        S->best_seqlen = P->seqlen;
        w->best_local = 1;
        w->version = G->g_version;
        o_backtrack(S, (uint32_t)(L - 1));
      } else {
        G->events[2]++;
        wm_adopt(w, G);
        w->best_local = 0;
        o_backtrack(S, (uint32_t)(L - 1));
        wm_recompare(w, P->level);
      }
      break;
    case 4:
      o_backtrack(S, (uint32_t)(L - 1));
      break;
    default:
      break;
  }
  wm_sync_auts(w, G);
}

/* other_path_node (sequential.cpp:304-392) with the prune rule */
static void wm_step(wm_worker* w, wm_shared* G) {
  osearch* S = &w->S;
  opart* P = &S->P;
  wm_sync_auts(w, G);
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
    ++G->nodes;
    P->seq[P->seqlen++] = v;
    o_individualize(P, v, &S->code, t->first);
    wm_classify(w, G);
    return;
  }
  /* worse than the private best and off the first path's trail */
  G->events[1]++;
  o_backtrack(S, P->level - 1);
  if (S->P.level >= 1) wm_recompare(w, S->P.level);
}

/* take item (k, v): 1 if started, 0 if its vertex is not the least of its orbit */
static int wm_start_item(wm_worker* w, wm_shared* G, uint32_t k, uint32_t v) {
  osearch* S = &w->S;
  opart* P = &S->P;
  int n = G->n;
  wm_copy_part(P, &G->leafP, n);
  P->level = G->D;
  o_reconstruct(P, k + 1, &S->eqlevfirst, &S->eqlevcanon, &S->comp_canon);
  P->level = k + 1;
  memcpy(P->seq, G->first_seq, (size_t)k * 4);
  P->seqlen = k;
  S->tc_level_reached = (int)k;
  o_select_tc(S);
  otc* t = &S->tcs[k];
  wm_sync_auts(w, G);
  t->last_num_aut = 0;
  if (S->num_aut > 0) o_orbits(S, t);
  t->last_num_aut = S->num_aut;
  if (t->elems[v] != (int32_t)v) return 0;
  t->counter = (uint32_t)n; /* no other child of the parent from this worker */
  if (w->version != G->g_version) wm_adopt(w, G);
  w->best_local = w->version == 0;
  for (uint32_t i = 0; i <= k; ++i) w->pathcode[i] = G->firstcode[i];
  S->eqlevfirst = k + 1;
  wm_recompare(w, k + 1);
  w->item_k = k;
  ++G->nodes;
  P->seq[P->seqlen++] = v;
  o_individualize(P, v, &S->code, t->first);
  wm_classify(w, G);
  return 1;
}

/* The worker hands over its shallowest untried child: the next orbit
 * representative of the target cell at the shallowest level of its item
 * below the item's own node, which it then treats as tried.  Only at levels
 * where a child's subtree is already finished (the path's child there is not
 * the cell's least vertex, the one tried first), so that the automorphisms
 * that subtree found prune the siblings before they are handed over. */
static int wm_donate(wm_worker* w, wm_shared* G, wm_gift* g) {
  osearch* S = &w->S;
  opart* P = &S->P;
  const int n = G->n;
  for (uint32_t Lp = w->item_k + 2; Lp < P->level && (int)Lp <= S->tc_level_reached; ++Lp) {
    otc* t = &S->tcs[Lp - 1];
    if (t->counter >= (uint32_t)n) continue;
    uint32_t least = (uint32_t)n;
    for (uint32_t x = 0; x < (uint32_t)n && least == (uint32_t)n; ++x)
      if (t->elems[x] >= 0) least = x;
    if (P->seq[Lp - 1] == least) continue; /* the first child is still running */
    if (S->num_aut > t->last_num_aut) {
      wm_sync_auts(w, G);
      /* orbits of the node at level Lp: automorphisms fixing its prefix */
      uint32_t saved = P->seqlen;
      P->seqlen = Lp - 1;
      o_orbits(S, t);
      P->seqlen = saved;
      t->last_num_aut = S->num_aut;
    }
    if (!o_next_rep(S, t)) continue;
    const uint32_t v = t->counter++;
    uint32_t e1 = 0xffffffffu;
    int e2 = 0x7fffffff, e3 = 0;
    wm_copy_part(&g->P, P, n);
    o_reconstruct(&g->P, Lp, &e1, &e2, &e3);
    g->P.level = Lp;
    g->L = Lp;
    memcpy(g->seq, P->seq, (size_t)(Lp - 1) * 4);
    memcpy(g->pathcode, w->pathcode, (size_t)Lp * sizeof(int));
    g->v = v;
    return 1;
  }
  return 0;
}

/* take a donated subtree: as an item whose parent is the gift's node */
static int wm_start_gift(wm_worker* w, wm_shared* G, const wm_gift* gf) {
  osearch* S = &w->S;
  opart* P = &S->P;
  const int n = G->n;
  const uint32_t k = gf->L - 1;
  if (G->replay) {
    /* as the GPU does: the first leaf back to the level the gift's sequence
     * shares with the first path, then its remaining vertices individualized
     * and refined, each code checked against the giver's */
    uint32_t c = 0;
    const uint32_t lim = k < G->D - 1 ? k : G->D - 1;
    while (c < lim && gf->seq[c] == G->first_seq[c]) ++c;
    wm_copy_part(P, &G->leafP, n);
    P->level = G->D;
    uint32_t e1 = 0xffffffffu;
    int e2 = 0x7fffffff, e3 = 0;
    o_reconstruct(P, c + 1, &e1, &e2, &e3);
    P->level = c + 1;
    memcpy(P->seq, G->first_seq, (size_t)c * 4);
    P->seqlen = c;
    for (uint32_t lvl = c + 1; lvl < gf->L; ++lvl) {
      int tc = -1;
      for (uint32_t i = 0; i < P->ncells; ++i)
        if (P->lcs[i].length > 1) {
          tc = (int)i;
          break;
        }
      if (tc < 0) {
        G->events[3]++;
        return 0;
      }
      const uint32_t u = gf->seq[lvl - 1];
      int code = 0;
      P->seq[P->seqlen++] = u;
      o_individualize(P, u, &code, P->lcs[tc].first);
      if (code != gf->pathcode[lvl]) G->events[3]++;
    }
  } else {
    wm_copy_part(P, &gf->P, n);
    P->level = gf->L;
    memcpy(P->seq, gf->seq, (size_t)k * 4);
    P->seqlen = k;
  }
  S->tc_level_reached = (int)k;
  o_select_tc(S);
  otc* t = &S->tcs[k];
  if (t->elems[gf->v] < 0) return 0;
  wm_sync_auts(w, G);
  t->last_num_aut = 0;
  if (S->num_aut > 0) o_orbits(S, t);
  t->last_num_aut = S->num_aut;
  if (t->elems[gf->v] != (int32_t)gf->v) return 0;
  t->counter = (uint32_t)n;
  if (w->version != G->g_version) wm_adopt(w, G);
  w->best_local = 0;
  memcpy(w->pathcode, gf->pathcode, (size_t)gf->L * sizeof(int));
  uint32_t e = 0;
  while (e < gf->L && e < G->D && w->pathcode[e] == G->firstcode[e]) ++e;
  S->eqlevfirst = e;
  wm_recompare(w, gf->L);
  w->item_k = k;
  ++G->nodes;
  P->seq[P->seqlen++] = gf->v;
  o_individualize(P, gf->v, &S->code, t->first);
  wm_classify(w, G);
  return 1;
}

int gcl_wide_model(int n, const int32_t* rowptr, const int32_t* col, const int32_t* color,
                   int workers, unsigned seed, int cap, int gate, int donate, uint8_t* out_nxn,
                   long* nodes_out, int* naut_out, long* events_out, uint32_t* auts_out,
                   long* rounds_out, uint32_t* first_seq_out) {
  if (n < 1 || workers < 1 || cap < 1) return -1;
  osearch S0;
  memset(&S0, 0, sizeof S0);
  S0.n = n;
  S0.max_aut = 1;
  if (o_alloc(&S0, n, 1)) return -1;
  opart* P = &S0.P;
  P->n = n;
  P->rp = rowptr;
  P->col = col;
  o_init_partition(P, color);
  S0.code = o_refine(P, NULL, 0);
  S0.firstcode[P->level - 1] = S0.code;
  wm_shared G;
  memset(&G, 0, sizeof G);
  G.n = n;
  G.cap = cap;
  G.replay = donate == 2;
  G.auts = malloc((size_t)cap * n * 4 + 4);
  G.nodes = 1;
  /* the first path, recording each level's target cell (sorted members) */
  uint32_t* tclen = calloc((size_t)n + 2, 4);
  uint32_t** tcm = calloc((size_t)n + 2, sizeof(uint32_t*));
  while (!o_discrete(P)) {
    o_select_tc(&S0);
    otc* t = &S0.tcs[S0.tc_level_reached - 1];
    uint32_t L = P->level;
    tclen[L - 1] = t->length;
    tcm[L - 1] = malloc((size_t)t->length * 4);
    uint32_t c = 0;
    for (int x = 0; x < n; ++x)
      if (t->elems[x] >= 0) tcm[L - 1][c++] = (uint32_t)x;
    uint32_t v = tcm[L - 1][0];
    ++G.nodes;
    P->seq[P->seqlen++] = v;
    o_individualize(P, v, &S0.code, t->first);
    S0.firstcode[P->level - 1] = S0.code;
  }
  G.D = P->level;
  G.firstcode = S0.firstcode;
  G.firstcode[G.D] = O_SENTINEL;
  G.first_seq = P->seq;
  G.first_seqlen = P->seqlen;
  G.first_label = malloc((size_t)n * 4);
  memcpy(G.first_label, P->elem, (size_t)n * 4);
  G.leafP = *P;
  G.g_code = malloc(((size_t)n + 2) * 4);
  for (uint32_t i = 0; i < G.D; ++i) G.g_code[i] = G.firstcode[i];
  G.g_code[G.D] = O_SENTINEL;
  G.g_level = (int)G.D;
  G.g_label = malloc((size_t)n * 4);
  memcpy(G.g_label, G.first_label, (size_t)n * 4);
  G.g_seq = malloc((size_t)n * 4 + 4);
  memcpy(G.g_seq, G.first_seq, (size_t)G.first_seqlen * 4);
  G.g_seqlen = G.first_seqlen;
  G.g_hash = malloc((size_t)n * n);
  o_leaf_matrix(&S0, G.g_hash);
  /* items, deepest level first */
  int tot = 0;
  for (uint32_t L = 1; L < G.D; ++L) tot += (int)tclen[L - 1] - 1;
  G.item_k = malloc(((size_t)tot + 1) * 4);
  G.item_v = malloc(((size_t)tot + 1) * 4);
  for (int L = (int)G.D - 1; L >= 1; --L)
    for (uint32_t j = 1; j < tclen[L - 1]; ++j) {
      G.item_k[G.nitems] = (uint32_t)(L - 1);
      G.item_v[G.nitems++] = tcm[L - 1][j];
    }
  wm_worker* ws = calloc((size_t)workers, sizeof(wm_worker));
  for (int i = 0; i < workers; ++i) {
    o_alloc(&ws[i].S, n, 1);
    free(ws[i].S.auts);
    ws[i].S.auts = G.auts;
    free(ws[i].S.subgroup);
    ws[i].S.subgroup = malloc((size_t)cap * sizeof(int) + 4);
    ws[i].S.n = n;
    ws[i].S.P.n = n;
    ws[i].S.P.rp = rowptr;
    ws[i].S.P.col = col;
    ws[i].pathcode = malloc(((size_t)n + 2) * 4);
    memcpy(ws[i].S.firstcode, G.firstcode, ((size_t)n + 2) * sizeof(int));
    memcpy(ws[i].S.first_seq, G.first_seq, (size_t)G.first_seqlen * 4);
    ws[i].S.first_seqlen = G.first_seqlen;
    memcpy(ws[i].S.first_label, G.first_label, (size_t)n * 4);
    ws[i].S.first_discovered = 1;
    ws[i].version = -1;
  }
  unsigned long long rs = 88172645463325252ull ^ (unsigned long long)seed;
  /* the level gate: an item starts once every item of the deeper levels is
   * done (need[it] = items before the first one of its level) */
  /* gate 2: on unless the levels hold fewer than 4 items each on average,
   * the GPU's automatic choice */
  const int probe = (gate & 8) != 0;
  gate &= 7;
  if (gate == 2) gate = G.nitems >= 4 * (int)(G.D > 1 ? G.D - 1 : 0);
  int* need = malloc(((size_t)G.nitems + 1) * sizeof(int));
  int* lfirst = malloc(((size_t)G.nitems + 1) * sizeof(int));
  int first = 0; /* the first item of the current level */
  for (int it = 0; it < G.nitems; ++it) {
    if (it == 0 || G.item_k[it] != G.item_k[it - 1]) first = it;
    need[it] = first;
    lfirst[it] = first;
  }
  long probe_start = -1; /* round the current level's probe started */
  int done = 0;
  long rounds = 0;
  /* donated subtrees waiting for a worker (at most one per idle worker) */
  wm_gift* gifts = calloc((size_t)workers, sizeof(wm_gift));
  for (int i = 0; i < workers; ++i) {
    gifts[i].P.elem = malloc((size_t)n * 4);
    gifts[i].P.lcs = malloc(((size_t)n + 1) * sizeof(ocell));
    gifts[i].seq = malloc((size_t)n * 4 + 4);
    gifts[i].pathcode = malloc(((size_t)n + 2) * sizeof(int));
  }
  int ngifts = 0;
#define WM_OPEN(it)                                                                         \
  (!gate || (done >= need[it] &&                                                            \
             (!probe || (it) == lfirst[it] || done > lfirst[it] ||                          \
              (probe_start >= 0 && rounds >= probe_start + 2 * (long)G.D))))
  for (int active = 1; active; ++rounds) {
    int idle = 0;
    const int items_open = G.next_item < G.nitems && WM_OPEN(G.next_item);
    for (int i = 0; i < workers; ++i) idle += !ws[i].busy && !items_open;
    for (int ii = 0; ii < workers; ++ii) {
      rs ^= rs << 13;
      rs ^= rs >> 7;
      rs ^= rs << 17;
      int i = seed ? (int)(rs % (unsigned long long)workers) : ii;
      wm_worker* w = &ws[i];
      if (w->busy) {
        wm_step(w, &G);
        if (w->S.P.level <= w->item_k + 1) {
          w->busy = 0;
          if (!w->gift) ++done;
        } else if (donate && ngifts < idle && wm_donate(w, &G, &gifts[ngifts])) {
          ++ngifts;
        }
      } else if (G.next_item < G.nitems && WM_OPEN(G.next_item)) {
        int it = G.next_item++;
        if (it == lfirst[it]) probe_start = rounds;
        w->gift = 0;
        if (wm_start_item(w, &G, G.item_k[it], G.item_v[it])) w->busy = w->S.P.level > w->item_k + 1;
        if (!w->busy) ++done;
      } else if (ngifts > 0) {
        wm_gift* gf = &gifts[--ngifts];
        w->gift = 1;
        if (wm_start_gift(w, &G, gf)) w->busy = w->S.P.level > w->item_k + 1;
      }
    }
    active = G.next_item < G.nitems || ngifts > 0;
    for (int i = 0; i < workers; ++i) active |= ws[i].busy;
  }
  for (int i = 0; i < workers; ++i) {
    free(gifts[i].P.elem);
    free(gifts[i].P.lcs);
    free(gifts[i].seq);
    free(gifts[i].pathcode);
  }
  free(gifts);
  free(need);
  free(lfirst);
  if (first_seq_out) memcpy(first_seq_out, G.first_seq, (size_t)G.first_seqlen * 4);
  if (rounds_out) {
    rounds_out[0] = rounds;
    rounds_out[1] = (long)G.D;
    rounds_out[2] = G.nitems;
  }
  if (out_nxn) memcpy(out_nxn, G.g_hash, (size_t)n * n);
  if (nodes_out) *nodes_out = G.nodes;
  if (naut_out) *naut_out = G.naut;
  if (events_out) memcpy(events_out, G.events, sizeof G.events);
  if (auts_out) memcpy(auts_out, G.auts, (size_t)G.naut * n * 4); /* cap x n entries */
  for (int i = 0; i < workers; ++i) {
    free(ws[i].pathcode);
    ws[i].S.auts = NULL; /* the shared store, freed below */
    o_free(&ws[i].S);
  }
  free(ws);
  for (int L = 0; L < n + 2; ++L) free(tcm[L]);
  free(tcm);
  free(tclen);
  free(G.auts);
  free(G.first_label);
  free(G.g_code);
  free(G.g_label);
  free(G.g_seq);
  free(G.g_hash);
  free(G.item_k);
  free(G.item_v);
  S0.max_aut = 1;
  o_free(&S0);
  return 0;
}

/* ---- exhaustive search: the maximum leaf over the whole tree ------------- */
typedef struct {
  int n;
  int* best_code;
  int best_level;
  uint8_t* best_hash;
  uint8_t* tmp_hash;
  int* path;
  long leaves, max_leaves;
  osearch* S;
} wm_exh;

static int wm_key_cmp(wm_exh* E, int L, const uint8_t* h) {
  for (int i = 0; i < L && i < E->best_level; ++i)
    if (E->path[i] != E->best_code[i]) return E->path[i] < E->best_code[i] ? -1 : 1;
  if (L < E->best_level) return 1;
  if (L > E->best_level) return -1;
  return o_cmp_upper(h, E->best_hash, E->n);
}

static void wm_exh_rec(wm_exh* E, opart* P) {
  int n = E->n;
  if (E->leaves > E->max_leaves) return;
  if (o_discrete(P)) {
    E->leaves++;
    opart saved = E->S->P;
    E->S->P = *P;
    o_leaf_matrix(E->S, E->tmp_hash);
    E->S->P = saved;
    int L = (int)P->level;
    if (E->best_level < 0 || wm_key_cmp(E, L, E->tmp_hash) > 0) {
      for (int i = 0; i < L; ++i) E->best_code[i] = E->path[i];
      E->best_level = L;
      memcpy(E->best_hash, E->tmp_hash, (size_t)n * n);
    }
    return;
  }
  int ci = -1;
  for (uint32_t i = 0; i < P->ncells; ++i)
    if (P->lcs[i].length > 1) {
      ci = (int)i;
      break;
    }
  ocell c = P->lcs[ci];
  uint32_t* mem = malloc((size_t)c.length * 4);
  memcpy(mem, P->elem + c.first, (size_t)c.length * 4);
  for (uint32_t j = 0; j < c.length; ++j) {
    opart Q = *P;
    Q.elem = malloc((size_t)n * 4);
    memcpy(Q.elem, P->elem, (size_t)n * 4);
    Q.lcs = malloc(((size_t)n + 1) * sizeof(ocell));
    memcpy(Q.lcs, P->lcs, ((size_t)n + 1) * sizeof(ocell));
    int code;
    o_individualize(&Q, mem[j], &code, c.first);
    E->path[Q.level - 1] = code;
    wm_exh_rec(E, &Q);
    free(Q.elem);
    free(Q.lcs);
  }
  free(mem);
}

/* 0 on success, 1 if the tree has more than max_leaves leaves */
int gcl_exhaustive_canon(int n, const int32_t* rowptr, const int32_t* col, const int32_t* color,
                         long max_leaves, uint8_t* out_nxn, long* leaves) {
  if (n < 1) return -1;
  osearch S0;
  memset(&S0, 0, sizeof S0);
  S0.n = n;
  if (o_alloc(&S0, n, 1)) return -1;
  opart* P = &S0.P;
  P->n = n;
  P->rp = rowptr;
  P->col = col;
  o_init_partition(P, color);
  wm_exh E;
  E.n = n;
  E.best_code = malloc(((size_t)n + 2) * 4);
  E.best_level = -1;
  E.best_hash = malloc((size_t)n * n);
  E.tmp_hash = malloc((size_t)n * n);
  E.path = malloc(((size_t)n + 2) * 4);
  E.leaves = 0;
  E.max_leaves = max_leaves;
  E.S = &S0;
  E.path[0] = o_refine(P, NULL, 0);
  wm_exh_rec(&E, P);
  int rc = E.leaves > max_leaves;
  if (!rc && out_nxn) memcpy(out_nxn, E.best_hash, (size_t)n * n);
  if (leaves) *leaves = E.leaves;
  free(E.best_code);
  free(E.best_hash);
  free(E.tmp_hash);
  free(E.path);
  o_free(&S0);
  return rc;
}
