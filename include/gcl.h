/* gcl.h -- C ABI of the B200 canonical-labeling library (libgcl_b200.so).
 *
 * The reference (rana-dbouk/gpu-canonical-labeling) has no FFI layer; its
 * boundary is the C++ entry points main.cpp calls:
 *
 *   std::vector<unsigned char> Nauty_Parallel(CSRGraph& graph, int max_aut,
 *       unsigned* node_count = nullptr, const std::string& prefix = "")
 *                                          -- src/nauty_parallel.h:9-13
 *   Nauty_Sequential(CSRGraph&, unsigned max_aut), result in
 *       best_leaf.hash_of_perm_graph       -- src/sequential.h:12-30
 *   canonical-form compare for the isomorphism verdict
 *                                          -- main.cpp:73-90, 172-197
 *
 * Every entry point here takes plain pointers and sizes.  Graphs are CSR with
 * both directions of every undirected edge stored and every row strictly
 * ascending (the shape CSRGraph::fromDIMACS builds, src/CSRGraph.cpp:40-119):
 * rowptr[n+1], col[rowptr[n]], optional color[n] (NULL = uncoloured).
 * Self loops, duplicate entries, unsorted rows (n > 64) and one-directional
 * edges are rejected with GCL_ERR_BAD_INPUT (the reference's refinement is
 * undefined on parallel edges).  Results are bit-identical to the reference's sequential
 * path: the canonical matrix, its best-leaf labeling, the number of stored
 * automorphisms and the number of search-tree nodes (the wide search of one
 * large graph keeps the matrix and has statistics of its own, see
 * GCL_OPT_WIDE_MIN_N).
 *
 * Errors are returned as negative status codes; nothing calls exit().  All
 * calls are synchronous unless named *_async; a synchronous call that fails
 * has no copy from or to the caller's buffers left in flight when it returns.
 * After GCL_ERR_NOMEM the context stays usable.  For tests of those paths,
 * GCL_FAULT_ALLOC_AT=k in the environment (k >= 1) makes the k-th device or
 * pinned host allocation of the process fail as out of memory, once.
 */
#ifndef GCL_H
#define GCL_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GCL_OK 0
#define GCL_ERR_ARG (-1)        /* bad argument (null pointer, n < 0, ...)  */
#define GCL_ERR_CUDA (-2)       /* CUDA runtime error                        */
#define GCL_ERR_NOMEM (-3)      /* device or host allocation failed          */
#define GCL_ERR_BAD_INPUT (-4)  /* loop / duplicate / asymmetric edge, index */
#define GCL_ERR_TOO_LARGE (-5)  /* graph above the supported vertex count    */
#define GCL_ERR_TIMEOUT (-6)    /* a bounded device wait ran out             */
#define GCL_ERR_INTERNAL (-7)

/* Per-graph status as written by the batched calls (out_status[g]). */
#define GCL_GRAPH_OK 0
#define GCL_GRAPH_BAD_INPUT 3
#define GCL_GRAPH_TOO_LARGE 2
#define GCL_GRAPH_INTERNAL 4  /* an internal consistency check failed: no result */
#define GCL_GRAPH_TIMEOUT 5   /* the graph's time budget (GCL_GRAPH_BUDGET_S, default
                                 600 s) ran out: no result                        */

/* Largest vertex count the library canonizes. */
#define GCL_MAX_N 65536

const char* gcl_status_string(int status);
int gcl_version(void);

/* ---- context ------------------------------------------------------------ */
/* A context owns device workspace, a stream and staging buffers on one GPU.
 * It is not thread-safe; use one context per host thread. */
typedef struct gcl_context gcl_context;

int gcl_create(int device, gcl_context** out);
int gcl_destroy(gcl_context* ctx);
/* The CUDA stream (cudaStream_t) the context launches on. */
void* gcl_stream(gcl_context* ctx);

/* ---- options -------------------------------------------------------------
 * GCL_OPT_WIDE_MIN_N: single-graph calls (gcl_canon_one, gcl_iso) on graphs
 *   with at least this many vertices use the wide search -- the search tree
 *   spread over every SM, like the reference's GPU path (a persistent grid of
 *   warps sharing one automorphism store and one best leaf).  Its canonical
 *   matrix is the sequential path's; its labeling is one of the equivalent
 *   best leaves and its statistics (stored automorphisms, nodes) are its own,
 *   as the reference GPU path's node count is.  Default 65 (the graphs the
 *   warp-per-graph kernel for n <= 64 does not take); GCL_MAX_N + 1 keeps the
 *   sequential traversal and its exact statistics for every size.  A wide
 *   search that fails for want of workspace falls back to the sequential one.
 * GCL_OPT_WORKSPACE_BYTES: device memory one pass of per-warp workspace may
 *   take (fewer resident warps when it binds); 0 = the GCL_WORKSPACE_GB
 *   environment variable, default 4 GiB.
 * GCL_OPT_WIDE_MAX_WARPS: upper bound on the warps of a wide search (0 = as
 *   many as fit on the GPU), to leave SMs to concurrent work.
 * GCL_OPT_SMEM_STAGE: 1 (default) lets the kernels for n > 64 keep their
 *   per-step arrays in shared memory (up to 200 KiB per block, which leaves
 *   little room on an SM for other kernels); 0 keeps them in device memory,
 *   for contexts whose long searches share the GPU with latency-bound work.
 * GCL_OPT_STREAM_PRIORITY: 1 replaces the context's stream by one of the
 *   highest priority (the block scheduler then starts its blocks before those
 *   of lower-priority streams), 0 by one of the lowest.  Waits for the
 *   context's work first; the stream gcl_stream returned before is gone.
 * GCL_OPT_WIDE_GATE: 1 (default) starts the wide search's items (the first
 *   path's siblings) level by level, deepest first, each level once the
 *   deeper ones are done, so their automorphisms prune it as in the
 *   sequential order; 0 starts every item at once, each testing its vertex
 *   against the automorphisms known at that moment.  Same canonical form
 *   either way.  0 suits searches whose levels hold few items each (trees:
 *   the gate runs their items one after another); it costs more nodes where
 *   levels are wide, and an orbit test per item over the whole store.  2
 *   chooses per search: off when the first path's levels hold fewer than 4
 *   items each on average, else on (decided on the device after the first
 *   path).  Every value gives the sequential canonical form in the GPU tests.
 * GCL_OPT_WIDE_SHARE: 1 lets a busy warp of the wide search hand an idle
 *   one an untried child below its first-path sibling -- at the shallowest
 *   level where a child's subtree has already finished, so that the
 *   automorphisms found there prune the siblings first -- through a device
 *   queue (up to 65,536 entries, 256 MiB); the receiver rebuilds the parent
 *   from the first leaf.  Same canonical form.  For trees whose work sits in
 *   a few siblings (unions of identical components: 6 copies of a random
 *   4-regular graph on 64 vertices in about 0.8 s on a B200, where the
 *   reference's sequential path takes 20.6 s on one core).  Default 0.
 * GCL_OPT_WIDE_PROBE: 1 (default) makes, under the level gate, the first
 *   item of each level run alone before the rest of that level starts, so
 *   the automorphisms it finds prune its siblings as they would in the
 *   sequential order (on vertex-transitive graphs such as tori one sibling
 *   per level covers the whole cell); 0 starts a level's items together.
 *   Same canonical form either way.
 * GCL_OPT_BATCH_HANDOFF_MS: t > 0 makes gcl_canon_batch give each graph of
 *   more than 64 vertices t ms in its batch warp; the graphs still searching
 *   then are searched again, one at a time, by the wide search (within the
 *   per-graph budget each and that budget in all).  Their canonical forms are
 *   the same; their labelings may be other equivalent best leaves and their
 *   statistics are the wide search's.  For mixed batches where a few graphs
 *   of large, symmetric or rigid families would hold the batch for minutes
 *   on one warp.  0 (default) off.
 * GCL_OPT_COUNTERS: 1 makes the wide searches of the context count events
 *   and clock cycles per part of the work (gcl_wide_counters), in a
 *   separately compiled items kernel; 0 (default) runs the kernel without
 *   them.  The counterpart of the reference's per-block section counters
 *   (src/structs.cuh:25-77), opt-in and without files.
 * GCL_OPT_BATCH_SPLIT: 1 makes gcl_canon_batch run a batch of at least
 *   4,096 graphs of up to 64 vertices as two halves, the second on a
 *   companion context with its own stream and workspace (created at the
 *   first such call, freed with the context): the second half's upload runs
 *   under the first half's kernels and the first half's results come back
 *   under the second half's kernels.  The results are the same.  0
 *   (default) runs the batch in one piece on the context's stream: on
 *   batches of small trees both halves end on their own longest searches
 *   at about the same time, and the split gained nothing measurable; two
 *   contexts driven from two host threads overlap whole calls instead.
 * Returns GCL_ERR_ARG for an unknown option or value. */
#define GCL_OPT_WIDE_MIN_N 1
#define GCL_OPT_WORKSPACE_BYTES 2
#define GCL_OPT_WIDE_MAX_WARPS 3
#define GCL_OPT_SMEM_STAGE 4
#define GCL_OPT_STREAM_PRIORITY 5
#define GCL_OPT_WIDE_GATE 6
#define GCL_OPT_WIDE_SHARE 7
#define GCL_OPT_COUNTERS 8
#define GCL_OPT_WIDE_PROBE 9
#define GCL_OPT_BATCH_HANDOFF_MS 10
#define GCL_OPT_BATCH_SPLIT 11
int gcl_set_option(gcl_context* ctx, int option, int64_t value);

/* Counters of the context's last wide search (gcl_canon_one on a graph of
 * at least GCL_OPT_WIDE_MIN_N vertices, gcl_canon_wide_device_async,
 * gcl_group_order), summed over the warps of its items kernel, when
 * GCL_OPT_COUNTERS was 1 for it.  Waits for the context's stream, writes up
 * to cap values to out and returns how many (16 in this version), or
 * GCL_ERR_ARG when that search was not counted.  In index order:
 *   0 items searched, 1 items pruned by an orbit, 2 handed-over subtrees
 *   taken, 3 subtrees handed over, 4 search-tree nodes, 5 leaves, 6
 *   automorphisms from the first leaf, 7 automorphisms from the best leaf, 8
 *   leaves that became the shared best, 9 publish retries after the shared
 *   best moved; clock cycles (clock64, summed over warps) 10 individualize +
 *   refine, 11 orbit tests, 12 waiting at the level gate, 13 waiting for a
 *   handed-over subtree, 14 leaf certificates and comparisons, 15 the warps'
 *   whole time in the kernel. */
int gcl_wide_counters(gcl_context* ctx, int64_t* out, int cap);

/* ---- one graph (drop-in for Nauty_Parallel, src/nauty_parallel.h:9-13) ---
 * out_nxn receives the n*n canonical adjacency matrix (row-major, 0/1 bytes,
 * canonical vertex i = row i), the value Nauty_Parallel returns.  node_count
 * and num_aut (either may be NULL) receive the search statistics.  ctx may be
 * NULL: a process-wide context on device 0 is created on first use (the
 * reference hard-codes device 0, src/nauty_parallel.cu:642-643); calls
 * through it from several threads take turns.  gcl_iso and gcl_group_order
 * take NULL the same way. */
int gcl_canon_one(gcl_context* ctx, const int32_t* rowptr, const int32_t* col,
                  const int32_t* color, int n, int max_aut, uint8_t* out_nxn,
                  int64_t* node_count, int64_t* num_aut);
/* The same with the canonical matrix bit-packed: out_rows receives n rows of
 * ceil(n/64) words, bit j of row i (word j/64, bit j%64) set iff canonical
 * vertices i and j are adjacent (gcl_canon_batch's out_rows), so a large
 * graph's result is n*n/8 bytes to copy and to read, not n*n. */
int gcl_canon_one_rows(gcl_context* ctx, const int32_t* rowptr, const int32_t* col,
                       const int32_t* color, int n, int max_aut, uint64_t* out_rows,
                       int64_t* node_count, int64_t* num_aut);

/* ---- batched: many graphs in one ragged CSR arena ----------------------
 * Graph g has n_g = voff[g+1]-voff[g] vertices; its local rowptr (n_g + 1
 * entries starting at 0) is at rowptr + voff[g] + g, its col entries at
 * col + eoff[g], its colours at color + voff[g] (color may be NULL).
 * Outputs (each may be NULL):
 *   out_dense + ooff[g]     n_g*n_g canonical matrix bytes
 *   out_rows + roff[g]      the same matrix bit-packed: n_g rows of
 *                           ceil(n_g/64) words, bit j of row i (word j/64,
 *                           bit j%64) set iff canonical vertices i and j are
 *                           adjacent -- equal exactly when the canonical
 *                           forms are equal, 8x smaller than out_dense
 *   out_label + voff[g]     best-leaf labeling, position -> vertex
 *   out_stats + 2*g         {num_aut, nodes}
 *   out_status[g]           GCL_GRAPH_* (required)
 * gcl_canon_batch takes HOST pointers and performs the copies; the _device
 * form takes DEVICE pointers and only enqueues work on the context stream
 * (call gcl_sync before reading results); it needs two host-side bounds:
 * max_n >= every n_g, and max_m2 >= every CSR entry count of a graph with
 * n_g > 64 (graphs up to 64 vertices never need it).  Both return GCL_OK when every
 * graph was processed, else the first failing graph's error. */
int gcl_canon_batch(gcl_context* ctx, int count, const int64_t* voff,
                    const int64_t* eoff, const int32_t* rowptr,
                    const int32_t* col, const int32_t* color, int max_aut,
                    uint8_t* out_dense, const int64_t* ooff, uint64_t* out_rows,
                    const int64_t* roff, int32_t* out_label, int64_t* out_stats,
                    int32_t* out_status);

int gcl_canon_batch_device_async(gcl_context* ctx, int count,
                                 const int64_t* d_voff, const int64_t* d_eoff,
                                 const int32_t* d_rowptr, const int32_t* d_col,
                                 const int32_t* d_color, int max_aut, int max_n,
                                 int64_t max_m2, uint8_t* d_out_dense,
                                 const int64_t* d_ooff, uint64_t* d_out_rows,
                                 const int64_t* d_roff,
                                 int32_t* d_out_label, int64_t* d_out_stats,
                                 int32_t* d_out_status);
int gcl_sync(gcl_context* ctx);

/* Batches whose arrays live in mapped host memory: gcl_host_alloc returns
 * pinned host memory of the context that its kernels can address (freed by
 * gcl_host_free or with the context).  gcl_canon_batch_mapped takes the
 * arguments of gcl_canon_batch, every array (inputs and outputs, whole)
 * inside such buffers, else GCL_ERR_ARG before any device work; for a batch
 * of graphs up to 64 vertices the kernels read the arena and write the
 * results in place over the bus, with no staging copies, so the transfers
 * overlap the search.  Batches with larger graphs (whose kernels read the CSR
 * again at every step) are copied as gcl_canon_batch does.  Synchronous.
 * Not yet measured on a GPU. */
int gcl_host_alloc(gcl_context* ctx, size_t bytes, void** out);
int gcl_host_free(gcl_context* ctx, void* ptr);
int gcl_canon_batch_mapped(gcl_context* ctx, int count, const int64_t* voff,
                           const int64_t* eoff, const int32_t* rowptr, const int32_t* col,
                           const int32_t* color, int max_aut, uint8_t* out_dense,
                           const int64_t* ooff, uint64_t* out_rows, const int64_t* roff,
                           int32_t* out_label, int64_t* out_stats, int32_t* out_status);

/* ---- one graph, wide search, device pointers --------------------------------
 * The wide search (see GCL_OPT_WIDE_MIN_N) of one graph already on the
 * device: rowptr[n+1], col[m], color[n] or NULL.  Outputs as in the batched
 * layout for a batch of one (each may be NULL except out_status[1]).  Work is
 * enqueued on the context stream; call gcl_sync before reading results. */
int gcl_canon_wide_device_async(gcl_context* ctx, const int32_t* d_rowptr,
                                const int32_t* d_col, const int32_t* d_color, int n,
                                int64_t m, int max_aut, uint8_t* d_out_dense,
                                uint64_t* d_out_rows, int32_t* d_out_label,
                                int64_t* d_out_stats, int32_t* d_out_status);

/* ---- batched, allocation-free (n <= 64) ---------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * where they canonize: a framework that owns all device memory through its
 * own allocator, a plugin in a process that forbids device allocations after
 * start-up, or a latency-critical path where an allocate/free pair would
 * synchronize the device.  Every pointer is a caller-owned DEVICE buffer in
 * the batched layout above; work is enqueued on `stream` (a cudaStream_t,
 * NULL = legacy default stream) of the current device and the call returns
 * without waiting.  Nothing is allocated: the per-warp scratch is one device
 * array of about 6.6 MiB that the library reserves statically on every GPU
 * it is loaded on, held until the process exits.
 *   Limits: max_n must be <= 64 (else GCL_ERR_TOO_LARGE, nothing launched);
 *   up to 128 stored automorphisms per graph when max_aut > 128 -- a graph
 *   that would store more reports GCL_GRAPH_AUT_OVERFLOW in out_status and
 *   no result.
 *   The first call on a device resolves the scratch's device address and the
 *   launch shape for that device; make that first call before any stream
 *   capture on the device.  That set-up is kept for the life of the process:
 *   after a cudaDeviceReset of a device, do not call this entry point on it
 *   again (the reset discards the array the kept address points into).
 *   All calls share the one scratch array, which keeps the last call's
 *   contents: calls that overlap on the GPU (other streams, other threads)
 *   race and corrupt each other; serialize them. */
#define GCL_GRAPH_AUT_OVERFLOW 1
int gcl_canon_batch_noalloc(void* stream, int count, const int64_t* d_voff,
                            const int64_t* d_eoff, const int32_t* d_rowptr,
                            const int32_t* d_col, const int32_t* d_color,
                            int max_aut, int max_n, uint8_t* d_out_dense,
                            const int64_t* d_ooff, int32_t* d_out_label,
                            int64_t* d_out_stats, int32_t* d_out_status);

/* ---- the reference's output text, written on the device -------------------
 * print_canonical_adjacency_list (main.cpp:33-70) for every graph of a batch,
 * from its bit-packed canonical rows (d_rows + d_roff[g]: n_g * ceil(n_g/64)
 * words, the out_rows layout of gcl_canon_batch_device_async) -- the text of
 * the reference's `output` file without an n x n byte matrix.  Two calls,
 * asynchronous on gcl_stream(ctx): with d_text NULL it writes the byte
 * offsets d_toff[count + 1] (d_toff[0] = 0); with d_text of d_toff[count]
 * bytes (read them back first) it writes graph g's text at d_text +
 * d_toff[g].  No reference counterpart as a call. */
int gcl_format_adjacency_device_async(gcl_context* ctx, int count, const int64_t* d_voff,
                                      const uint64_t* d_rows, const int64_t* d_roff,
                                      int64_t* d_toff, char* d_text);

/* ---- files: DIMACS parsing overlapped with the GPU -------------------------
 * Canonize `count` DIMACS files (the reference's graph.txt format,
 * CSRGraph::fromDIMACS, src/CSRGraph.cpp:40-119) in chunks of `chunk` files
 * (0 = 4096): `threads` host threads (0 = all cores) parse chunk k while the
 * GPU canonizes chunk k-1 through the batched path.  For every file, in
 * order and on the calling thread, cb receives its index, a GCL_GRAPH_*
 * status (an unreadable file, an endpoint out of range or a duplicate edge
 * is GCL_GRAPH_BAD_INPUT, more than GCL_MAX_N vertices GCL_GRAPH_TOO_LARGE),
 * n, the packed canonical rows (n * ceil(n/64)
 * words) and the labeling -- both NULL unless the status is GCL_GRAPH_OK,
 * valid only during the call -- and the statistics.  Returns GCL_OK once
 * every file has been delivered, else the first launch or copy error. */
typedef void (*gcl_file_result_fn)(void* user, int64_t index, int32_t status, int n,
                                   const uint64_t* rows, const int32_t* label,
                                   int64_t num_aut, int64_t nodes);
int gcl_canon_files(gcl_context* ctx, int64_t count, const char* const* paths, int max_aut,
                    int chunk, int threads, gcl_file_result_fn cb, void* user);

/* ---- autotuning of the batched launches ----------------------------------
 * The batched path runs the warp kernel (n <= 64) and one sparse-kernel pass
 * per size bucket (n <= 256, <= 1024, <= 4096, larger).  gcl_autotune times
 * them on a sample batch (host arrays in the batched layout) under candidate
 * launch shapes -- resident blocks per SM of the warp kernel; per sparse
 * bucket, shared-memory staging on or off and resident blocks per SM --
 * keeps for each the fastest, applies the choice to the context and returns
 * it.  A bucket without graphs in the sample keeps its default (its sp_ms is
 * -1).  Results are unchanged by any choice: only the launch shape moves.
 * gcl_set_tuning applies a saved choice (0 / -1 fields = default). */
typedef struct {
  int w64_blocks_per_sm;    /* 0 = as many as fit                           */
  int sp_blocks_per_sm[4];  /* 0 = as many as fit                           */
  int sp_stage[4];          /* 1 = stage in shared memory, 0 = not, -1 = default */
  float w64_ms;             /* best pass time found (ms), -1 = not timed    */
  float sp_ms[4];
} gcl_tuning;
int gcl_autotune(gcl_context* ctx, int count, const int64_t* voff, const int64_t* eoff,
                 const int32_t* rowptr, const int32_t* col, const int32_t* color,
                 int max_aut, int repeats, gcl_tuning* out);
int gcl_set_tuning(gcl_context* ctx, const gcl_tuning* tuning);

/* ---- automorphism group order --------------------------------------------
 * The reference never computes |Aut(G)|; it prints how many automorphisms it
 * stored (sequential.cpp:83), which depends on the traversal and max_aut.
 * gcl_group_order runs the wide search with a store that keeps every
 * automorphism found.  The first path's individualized vertices are a base
 * of Aut(G) and those automorphisms a strong generating set for it, so the
 * order is the product over the first path of each vertex's orbit under the
 * stored automorphisms that fix the vertices before it (nauty's grpsize).
 * The host checks it with the Schreier-Sims completion (general, then on that
 * base), whose order is returned when one finishes within its work budget
 * (about a second).  *log10_order = log10 |Aut|,
 * digits (if not NULL) the order in decimal, *generators the automorphisms
 * the search stored, *checked (if not NULL) how the order was confirmed:
 * 1 a finished Schreier-Sims completion gave the same order; -1 it gave a
 * different one, which is returned (the stored automorphisms generate the
 * group but are no strong generating set for the first path); 0 neither
 * completion finished within its budget and the orbit product is returned
 * unchecked.  GCL_ERR_TOO_LARGE if the search found more
 * automorphisms than its 1 GiB store holds, GCL_ERR_ARG if digits_cap is too
 * small.  gcl_perm_group_order returns GCL_ERR_TIMEOUT when its
 * Schreier-Sims exceeds the work cap.
 * gcl_perm_group_order is the host part alone: the order of the group
 * generated by `count` permutations of {0..n-1} (row a at perms + a*n). */
int gcl_group_order(gcl_context* ctx, const int32_t* rowptr, const int32_t* col,
                    const int32_t* color, int n, double* log10_order, char* digits,
                    int digits_cap, int64_t* generators, int* checked);
int gcl_perm_group_order(int n, const uint16_t* perms, int64_t count, double* log10_order,
                         char* digits, int digits_cap);

/* ---- isomorphism (main.cpp:172-197) --------------------------------------
 * *verdict = 1 when the canonical upper triangles are equal (ISOMORPHIC),
 * 0 otherwise.  Graphs with different vertex counts are NOT ISOMORPHIC (the
 * reference compares n1 x n1 entries and reads out of bounds when n2 < n1). */
int gcl_iso(gcl_context* ctx, const int32_t* rowptr1, const int32_t* col1,
            const int32_t* color1, int n1, const int32_t* rowptr2,
            const int32_t* col2, const int32_t* color2, int n2, int max_aut,
            int* verdict);

/* ---- serving: a request loop with continuous batching -------------------
 * No counterpart in the reference (its CLI canonizes one or two graphs per
 * process).  A server owns `lanes` device contexts, each with its own stream
 * and workspace; one dispatcher thread keeps every lane busy: whenever a lane
 * is free it takes the queued requests that fit the lane's device-memory
 * budget (graphs, outputs and search workspace -- admission by HBM
 * footprint) and launches them as one batch, so requests that arrive while
 * others are on the GPU run in the next batch on another lane, overlapping
 * on the device.  Requests are split in four classes by their largest
 * graph -- small (n < mid_n: the warp kernel for n <= 64), mid, big, and
 * large (n >= large_n: the wide search, one request at a time, one block per
 * SM) -- each with its own queue, lanes and batch-size cap, so a batch
 * never waits for a slower class.  Results are those of
 * gcl_canon_batch (gcl_canon_wide_device_async for large) on the same graph.
 *
 * After each batch a kernel hashes every canonical form into a device table
 * (open addressing, 64-bit keys, forms kept in a device store and compared in
 * full on a key match): equal class ids mean isomorphic graphs, and a
 * request whose class was seen before is reported as a repeat.  Exact
 * repeats of an earlier input are answered from a host-side memo of recent
 * results without a launch.
 *
 * Thread safety: submit, poll and stats may be called from any threads.
 *
 * Each lane is a CUDA stream.  Streams beyond CUDA_DEVICE_MAX_CONNECTIONS
 * (default 8) share hardware work queues, and a short batch then waits
 * behind a long search that happens to share its queue: set the variable to
 * at least the number of lanes (32 is the maximum) before the process
 * first uses CUDA. */
typedef struct gcl_server gcl_server;

typedef struct {
  int lanes;           /* lanes for requests whose graphs have n < mid_n, default 3 */
  int mid_lanes;       /* lanes for mid_n <= n < big_n, default 3              */
  int big_lanes;       /* lanes for big_n <= n < large_n, default 8            */
  int large_lanes;     /* lanes for n >= large_n (wide search), default 4      */
  int max_batch;       /* graphs per small batch, default 8192                */
  int mid_batch;       /* graphs per mid batch, default 512                   */
  int big_batch;       /* graphs per big batch, default 8                     */
  int mid_n;           /* default 65                                          */
  int big_n;           /* default 257                                         */
  int large_n;         /* default 2049                                        */
  int max_aut;         /* default 10000                                       */
  int64_t lane_bytes;  /* device-memory budget of one batch (inputs, outputs,
                          search workspace) on the batched lanes, 256 MiB      */
  int64_t table_slots; /* canonical-hash table slots (power of two), 1 << 20  */
  int64_t store_bytes; /* device store of canonical forms, default 256 MiB    */
  int64_t memo_bytes;  /* host memo of exact repeats, default 64 MiB, < 0 = off */
  int big_wide;        /* 1: the big lanes run each request through the wide
                          search, one request at a time on up to 128 warps,
                          and every wide search picks its level gate per graph
                          (GCL_OPT_WIDE_GATE 2); a wide search that runs out
                          of orbit storage is rerun on a mid lane.  Default 0:
                          the batched sequential search.  Not yet measured on
                          a GPU.                                               */
} gcl_serve_config;

#define GCL_REQ_CANON 0
#define GCL_REQ_ISO 1

typedef struct {
  int64_t id;          /* the id given to gcl_serve_submit                      */
  int32_t status;      /* GCL_OK or a GCL_ERR_* code                           */
  int32_t verdict;     /* GCL_REQ_ISO: 1 isomorphic, 0 not; else -1            */
  int32_t repeat;      /* 1: an isomorphic graph was canonized before (the
                          class was in the table); 2: an identical input was
                          answered from the memo                               */
  int32_t batch;       /* graphs in the batch that carried the request (0 = memo) */
  int64_t class_id;    /* isomorphism class of (the first) graph, -1 unknown   */
  uint64_t canon_hash; /* 64-bit hash of the canonical form                    */
  double latency_s;    /* submit -> result ready (host steady clock)           */
  /* the request's timeline, seconds after submit like latency_s (0 for a
     memo answer): taken into a batch, the batch's work enqueued on its lane
     (copies, kernels), and the lane's stream reached the batch's end on the
     GPU (its completion callback ran) */
  double admit_s, launch_s, gpu_done_s;
} gcl_serve_result;

typedef struct {
  int64_t submitted, completed, batches, graphs, memo_hits, class_repeats, classes;
  int64_t large_graphs;
  /* per request class (small, mid, big, large): batches launched, their
     summed launch-to-result time and summed time queued before launch (ns) */
  int64_t class_batches[4], class_batch_ns[4], class_queue_ns[4];
  /* per request class: the longest host time the dispatcher spent enqueuing
     one batch (packing, copies and launches issued) and finishing one
     (results handed out), ns -- the dispatcher serves every lane, so this is
     time no other lane could be launched or finished */
  int64_t class_max_launch_ns[4], class_max_complete_ns[4];
  /* the longest host time of each part of enqueuing one batch, over all
     batches (ns): pinned host buffers grown, device buffers grown, requests
     packed, copies in issued, the search launched, the table kernel and the
     copies out issued */
  int64_t enqueue_part_max_ns[6];
} gcl_serve_stats;

/* cfg may be NULL (all defaults); zero fields take their default. */
int gcl_serve_create(int device, const gcl_serve_config* cfg, gcl_server** out);
/* Waits for work in flight, then frees everything. */
int gcl_serve_destroy(gcl_server* srv);
/* Queue a request.  The graphs are copied before the call returns.  For
 * GCL_REQ_CANON the second graph is ignored and out_rows (n * ceil(n/64)
 * words, the packed layout of gcl_canon_batch) and out_label (n) may be
 * NULL or caller buffers that stay valid until the request's result has been
 * polled.  For GCL_REQ_ISO both outputs are ignored. */
int gcl_serve_submit(gcl_server* srv, int64_t id, int kind, const int32_t* rowptr,
                     const int32_t* col, const int32_t* color, int n,
                     const int32_t* rowptr2, const int32_t* col2, const int32_t* color2,
                     int n2, uint64_t* out_rows, int32_t* out_label);
/* Up to max finished results; waits up to timeout_ms (0 = do not wait, -1 =
 * until at least one is ready).  Returns the number written or an error. */
int gcl_serve_poll(gcl_server* srv, gcl_serve_result* out, int max, int timeout_ms);
int gcl_serve_stats_get(gcl_server* srv, gcl_serve_stats* out);

/* Open-loop load: request i (kind[i], graphs g1[i] and g2[i] of the arena in
 * the batched layout) is submitted at arrival_s[i] seconds after the call
 * starts, from a generator thread, whatever the server's progress; the call
 * returns when every result is in (results[i] for request i, latency
 * measured from the scheduled arrival) or timeout_s has passed
 * (GCL_ERR_TIMEOUT). */
int gcl_serve_replay(gcl_server* srv, int nreq, const double* arrival_s, const int32_t* kind,
                     const int32_t* g1, const int32_t* g2, int count, const int64_t* voff,
                     const int64_t* eoff, const int32_t* rowptr, const int32_t* col,
                     const int32_t* color, double timeout_s, gcl_serve_result* results);

#ifdef __cplusplus
}
#endif
#endif /* GCL_H */
