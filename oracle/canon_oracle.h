/* canon_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's sequential individualization-refinement
 * canonical labeler (src/sequential.cpp, src/partition_refinement.cpp,
 * src/perm_group.cpp).  Used by tests/ as the parity oracle, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline leg.  The product
 * library never links or calls it.
 *
 * Parity pin: tests/test_oracle.py checks this restatement against the golden
 * fixtures in tests/golden/ (generated by running the reference's own
 * sequential code, compiled from its sources by oracle/Makefile `ref`) and,
 * where oracle/_ref/libgcl_ref.so is present, against the reference directly
 * on fresh seeded graphs.
 */
#ifndef GCL_CANON_ORACLE_H
#define GCL_CANON_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int64_t num_aut; /* automorphisms stored (sequential.cpp:83)          */
  int64_t nodes;   /* search tree nodes created (sequential.cpp:85)     */
} gcl_oracle_stats;

/* Canonical form of one graph.  rowptr[n+1]/col: CSR with both directions,
 * sorted rows, no loops, no duplicates; color[n] or NULL.  out_nxn (n*n
 * bytes, may be NULL) receives the canonical adjacency matrix, label_out
 * (n ints, may be NULL) the best leaf's vertex order (position -> vertex).
 * Returns 0, or -1 on bad arguments / allocation failure. */
int gcl_oracle_canon(int n, const int32_t* rowptr, const int32_t* col,
                     const int32_t* color, unsigned max_aut, uint8_t* out_nxn,
                     int32_t* label_out, gcl_oracle_stats* st);

/* Same over a ragged arena (layout of graphs.Arena): graph g has n_g =
 * voff[g+1]-voff[g] vertices, rowptr at rowptr_arena + voff[g] + g, col at
 * col_arena + eoff[g], colours at color_arena + voff[g] (NULL = none).
 * out_arena + ooff[g] receives n_g*n_g bytes when out_arena != NULL;
 * label_arena + voff[g] receives the label when label_arena != NULL. */
int gcl_oracle_canon_batch(int count, const int64_t* voff, const int64_t* eoff,
                           const int32_t* rowptr_arena, const int32_t* col_arena,
                           const int32_t* color_arena, unsigned max_aut,
                           uint8_t* out_arena, const int64_t* ooff,
                           int32_t* label_arena, gcl_oracle_stats* stats);

/* Root refinement only: the equitable partition of the colour partition
 * (partition_refinement.cpp:28-68 then :150-485 with every cell active).
 * elem_out[n] = element order, cell_start_out[n] = start position of the
 * cell containing each position, returns the refinement code. */
int gcl_oracle_root_refine(int n, const int32_t* rowptr, const int32_t* col,
                           const int32_t* color, int32_t* elem_out,
                           int32_t* cell_start_out);

#ifdef __cplusplus
}
#endif
#endif
