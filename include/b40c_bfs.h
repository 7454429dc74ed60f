/*
 * b40c_bfs.h -- C ABI of libb40c_bfs.so, a B200 (sm_100a) breadth-first search
 * that stands in for b40c::graph::bfs of back40computing (b40c v1.0.1042).
 *
 * Every entry point returns an int whose value is a cudaError_t code
 * (0 = success), the way every reference method returns cudaError_t.  The
 * message of the last failure on the calling thread is available from
 * b40c_last_error_string().  Signatures use plain pointers and sizes only.
 *
 * Reference interfaces are cited as file:line inside the back40computing tree.
 */
#ifndef B40C_BFS_H
#define B40C_BFS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes (numeric values of cudaError_t) ----------------------- */
#define B40C_SUCCESS                      0
#define B40C_ERR_INVALID_VALUE            1    /* cudaErrorInvalidValue */
#define B40C_ERR_MEMORY_ALLOCATION        2    /* cudaErrorMemoryAllocation */
#define B40C_ERR_INVALID_CONFIGURATION    9    /* cudaErrorInvalidConfiguration: frontier queue overflow
                                                  (enactor_contract_expand.cuh:318-324) */
#define B40C_ERR_INVALID_DEVICE_FUNCTION  98   /* cudaErrorInvalidDeviceFunction */
#define B40C_ERR_ILLEGAL_STATE            401  /* cudaErrorIllegalState: call out of order */
#define B40C_ERR_LAUNCH_TIMEOUT           702  /* cudaErrorLaunchTimeout: a bounded device wait gave up */
#define B40C_ERR_NOT_SUPPORTED            801  /* cudaErrorNotSupported */

/* ---- enumerations -------------------------------------------------------- */
/* FrontierType, b40c/graph/bfs/csr_problem.cuh:54-61 */
#define B40C_VERTEX_FRONTIERS     0
#define B40C_EDGE_FRONTIERS       1
#define B40C_MIXED_FRONTIERS      2
#define B40C_MULTI_GPU_FRONTIERS  3

/* Strategy, test/bfs/test_bfs.cu:71-78 (MULTI_GPU is not provided) */
#define B40C_EXPAND_CONTRACT  0
#define B40C_CONTRACT_EXPAND  1
#define B40C_TWO_PHASE        2
#define B40C_HYBRID           3

/* Which enact method: EnactSearch / EnactFusedSearch / EnactIterativeSearch */
#define B40C_VARIANT_DEFAULT    0
#define B40C_VARIANT_FUSED      1
#define B40C_VARIANT_ITERATIVE  2

typedef struct b40c_problem b40c_problem_t;   /* bfs::CsrProblem<int,int,MARK_PREDECESSORS> */
typedef struct b40c_enactor b40c_enactor_t;   /* bfs::Enactor{ContractExpand,ExpandContract,TwoPhase,Hybrid} */

/* ---- library ------------------------------------------------------------- */
/* Message of the last failure on this thread ("" if none). */
const char *b40c_last_error_string(void);
/* Library version string. */
const char *b40c_version(void);

/* ---- CsrProblem (b40c/graph/bfs/csr_problem.cuh:68-751) ------------------ */
/* CsrProblem() ctor (:229-233), on the current CUDA device.  mark_predecessors
 * selects the MARK_PREDECESSORS template flag (:66). */
int b40c_problem_create(int mark_predecessors, b40c_problem_t **out);
/* ~CsrProblem (:240-249) and GraphSlice::~GraphSlice (:152-172). */
int b40c_problem_destroy(b40c_problem_t *problem);
/* FromHostProblem(stream_from_host, nodes, edges, h_column_indices,
 * h_row_offsets, num_gpus) (:328-403).  The host CSR stays caller-owned; it is
 * validated (monotone offsets, ids in range) and copied to the device.
 * stream_from_host maps the host arrays instead (they must be pinned and
 * mapped, or are registered here).  num_gpus must be <= 1. */
int b40c_problem_from_host(b40c_problem_t *problem, int stream_from_host,
                           int nodes, int edges,
                           const int *h_column_indices, const int *h_row_offsets,
                           int num_gpus);
/* Reset(frontier_type, queue_sizing) (:547-750): lazily (re)allocates the
 * frontier queues, sets labels := -1 and the visited mask := 0; synchronous. */
int b40c_problem_reset(b40c_problem_t *problem, int frontier_type, double queue_sizing);
/* Same, but only enqueues the label/mask initialisation on the problem's
 * stream (allocation, when needed, is still done before returning). */
int b40c_problem_reset_async(b40c_problem_t *problem, int frontier_type, double queue_sizing);
/* ExtractResults(h_label) (:255-273): copies nodes labels to the host. */
int b40c_problem_extract_results(b40c_problem_t *problem, int *h_labels);
/* Enqueues the label copy on the problem's stream without waiting.  With two
 * label buffers (below) the copy goes to a side stream instead; wait for it
 * with b40c_problem_sync. */
int b40c_problem_extract_results_async(b40c_problem_t *problem, int *h_labels);
/* No reference counterpart (the reference keeps one d_labels array,
 * csr_problem.cuh:116).  count = 2: each Reset switches between two label
 * arrays, and ExtractResultsAsync copies the last search's labels on a side
 * stream, so that copy overlaps the next Reset and search; the device label
 * pointer (b40c_problem_info) then changes with every Reset.  count = 1 (the
 * default): one array, as in the reference.  Costs 4 bytes per vertex more. */
int b40c_problem_set_label_buffers(b40c_problem_t *problem, int count);
/* Waits for all work queued on the problem: its stream and side-stream label
 * copies. */
int b40c_problem_sync(b40c_problem_t *problem);
/* 8-byte vertex ids with int sizes, the reference's g500 configuration
 * (VertexId = long long, SizeT = int; test/bfs/test_bfs.cu:1068-1093):
 * the column ids are checked and narrowed to the device's int32 layout (every
 * id of a graph with int sizes fits), labels are widened on the way out.
 * stream_from_host is not available with 8-byte ids (cudaErrorNotSupported). */
int b40c_problem_from_host_ids64(b40c_problem_t *problem, int stream_from_host, int nodes, int edges,
                                 const long long *h_column_indices, const int *h_row_offsets, int num_gpus);
int b40c_problem_extract_results_ids64(b40c_problem_t *problem, long long *h_labels);
/* nodes, edges and the GraphSlice device pointers (:99-173). Any out pointer may be NULL. */
int b40c_problem_info(b40c_problem_t *problem, int64_t *nodes, int64_t *edges,
                      void **d_row_offsets, void **d_column_indices,
                      void **d_labels, void **d_visited_mask);
/* CUDA device ordinal the problem lives on (GraphSlice::gpu, :103). */
int b40c_problem_device(b40c_problem_t *problem, int *device);
/* Stream (a cudaStream_t) for every later operation on this problem; NULL = the
 * library's own stream for this problem. */
int b40c_problem_set_stream(b40c_problem_t *problem, void *stream);

/* ---- Enactors (b40c/graph/bfs/enactor_*.cuh) ----------------------------- */
/* Enactor{ExpandContract,ContractExpand,TwoPhase,Hybrid}<INSTRUMENT>(DEBUG)
 * ctor (enactor_expand_contract.cuh:~200, enactor_contract_expand.cuh:206-214,
 * enactor_two_phase.cuh:221-229, enactor_hybrid.cuh:64). */
int b40c_enactor_create(int strategy, int instrument, int debug, b40c_enactor_t **out);
int b40c_enactor_destroy(b40c_enactor_t *enactor);
/* GetFrontierType() (enactor_base.cuh:72). */
int b40c_enactor_frontier_type(b40c_enactor_t *enactor, int *frontier_type);
/* EnactSearch / EnactFusedSearch / EnactIterativeSearch(problem, src,
 * max_grid_size) (enactor_contract_expand.cuh:259-407, :416-596;
 * enactor_expand_contract.cuh:258-373; enactor_two_phase.cuh:416-765;
 * enactor_hybrid.cuh:279-560).  Synchronous: returns after the search, with
 * cudaErrorInvalidConfiguration on frontier overflow. */
int b40c_enact_search(b40c_enactor_t *enactor, b40c_problem_t *problem,
                      int src, int max_grid_size, int variant);
/* Enqueues the search on the enactor's stream and returns; overflow and
 * barrier-timeout flags are checked by the next b40c_enactor_sync. */
int b40c_enact_search_async(b40c_enactor_t *enactor, b40c_problem_t *problem,
                            int src, int max_grid_size, int variant);
/* Waits for the enactor's stream and reports flags raised by async searches. */
int b40c_enactor_sync(b40c_enactor_t *enactor);
/* GetStatistics(total_queued, search_depth, avg_duty)
 * (enactor_contract_expand.cuh:237-250).  search_depth = iteration - 1.
 * With INSTRUMENT: total_queued sums the levels' input frontiers, and
 * avg_duty (fused searches) is the CTAs' time in level work -- barrier waits
 * excluded -- over the longest CTA's time times the grid, as the reference's
 * KernelRuntimeStats accumulate it (1.0: perfectly balanced levels); else 0. */
int b40c_enactor_get_statistics(b40c_enactor_t *enactor, long long *total_queued,
                                int *search_depth, double *avg_duty);
/* Device time of the last synchronous search (CUDA events around its kernels). */
int b40c_enactor_last_elapsed_ms(b40c_enactor_t *enactor, float *ms);
/* Stream (a cudaStream_t) for later searches; NULL = the enactor's own stream. */
int b40c_enactor_set_stream(b40c_enactor_t *enactor, void *stream);
/* Tuning policy (the reference's compile-time KernelPolicy, kernel_policy.cuh:61-87,
 * WARP_GATHER_THRESHOLD / CTA_GATHER_THRESHOLD): cta_threads in {128,256,512}
 * (default 512 for expand-contract, 256 for the others);
 * lists of at least cta_gather_threshold edges (default 1024) are cut into
 * chunks of 16 * cta_threads edges, each gathered by a whole CTA; lists of at
 * least warp_gather_threshold edges (default 128 for expand-contract, 64 for
 * the others) into chunks of 512 edges,
 * each gathered by one warp; chunks are shared by the whole grid; shorter
 * lists are gathered by a warp prefix sum.  cull_flags: bit0 warp-level cull
 * (__match_any_sync), bit1 history cull through a per-CTA shared-memory cache
 * of visited-mask words (default: bit1 only).  A 0 keeps a threshold, a -1
 * keeps the cull flags. */
int b40c_enactor_set_policy(b40c_enactor_t *enactor, int cta_threads,
                            int warp_gather_threshold, int cta_gather_threshold, int cull_flags);
/* Per-level log (the reference's DEBUG per-level queue lengths,
 * enactor_two_phase.cuh:496-499, with device timestamps): when enabled, each
 * later search records per level its %globaltimer start, its input frontier
 * queue length and its input CTA and warp chunk counts. */
int b40c_enactor_set_level_log(b40c_enactor_t *enactor, int enable);
/* Copies up to max_records records of the last search (any out pointer may be
 * NULL); *count gets the number copied, the last one being the end marker
 * (all counts 0).  frontier counts queued vertices (edge-frontier strategies:
 * queued edges); lists long enough to be cut into chunks are counted in
 * chunks / wchunks instead; bottom_up is 1 for a level that ran bottom-up.
 * Levels of the two-phase strategy are its phases. */
int b40c_enactor_level_log(b40c_enactor_t *enactor, int max_records, int64_t *t_start_ns,
                           int *frontier, int *chunks, int *wchunks, int *bottom_up, int *count);
/* The level log's times (same records as b40c_enactor_level_log): each
 * phase's start and the moment the last CTA finished its work, before the
 * grid barrier that ends it (0 for per-level launches and the end marker);
 * the gap to the next start is the barrier's cost.  No counterpart in the
 * reference. */
int b40c_enactor_level_times(b40c_enactor_t *enactor, int max_records, int64_t *t_start_ns,
                             int64_t *t_work_end_ns, int *count);
/* Direction-optimizing expand-contract (an addition; the reference's
 * expand-contract is top-down only): a level runs bottom-up -- each unvisited
 * vertex scans its list for a parent in the frontier -- once the frontier's
 * edges exceed the unvisited vertices' edges / alpha, and returns to top-down
 * once the frontier holds fewer than nodes / beta vertices and shrinks
 * (Beamer, Asanovic and Patterson, SC 2012).  Defaults alpha = 14, beta = 24;
 * alpha = 0 turns it off.  It applies to fused searches on symmetric graphs
 * held on the device (not stream_from_host), checked once per graph; other
 * searches stay top-down.  Depth
 * labels, search depth and total_queued are those of top-down; predecessor
 * labels are valid predecessors (bottom-up levels record the parent they
 * find). */
int b40c_enactor_set_direction_optimizing(b40c_enactor_t *enactor, int alpha, int beta);
/* Spin limit of every device-side wait (grid barrier), in microseconds. */
int b40c_enactor_set_wait_limit_us(b40c_enactor_t *enactor, long long us);
/* L2 residency of the search state (no counterpart in the reference, which
 * reads the visited mask through the texture cache, contract_expand_atomic/
 * cta.cuh:213-258): what = 0 off (the default), 1 the visited mask, 2 the
 * visited mask and the labels.  The enactor sets a persisting access-policy
 * window on its stream for its own launches and clears it after them; the
 * first use sets the context's persisting-L2 limit
 * (cudaLimitPersistingL2CacheSize, which ends with the process) to the
 * window's size, within the device maximum. */
int b40c_enactor_set_l2_persistence(b40c_enactor_t *enactor, int what);
/* Bottom-up levels of direction-optimizing searches stage each step's row
 * offsets, heaviest-neighbour keys and visited-mask words in shared memory
 * with bulk copies issued one step ahead (enable = 1, where the kernel's
 * shared memory allows it: 512-thread CTAs, depth labels), or load them when
 * the step starts (0, the default: on R-MAT scale 22 the stage buffers' share
 * of each SM's shared memory and L1 costs more than the copies save).
 * Results are the same either way.  No
 * counterpart in the reference, which reads row offsets per tile through the
 * texture path (contract_expand_atomic/cta.cuh:187-207). */
int b40c_enactor_set_bottom_up_staging(b40c_enactor_t *enactor, int enable);
/* Narrow levels (fused searches of every strategy; per-level launches ignore
 * it), for high-diameter graphs (lattices, road networks), whose levels are a
 * few thousand edges and whose search time is mostly the latency of each
 * level:
 *  - the levels whose input is a frontier (edges, or vertices for
 *    expand-contract) of at most max_frontier queued entries, without lists
 *    long enough to be cut into chunks, and, for expand-contract, that the
 *    direction switch keeps top-down, run (two-phase: both phases of each)
 *    from the source on ONE thread-block cluster of team_ctas CTAs (at most
 *    16, fewer when the device cannot co-schedule that many), whose levels
 *    end at the cluster's hardware barrier; the first larger level and all
 *    after it run on the full persistent grid (team_ctas = 0: all do; the
 *    hybrid's bound is at most its contract-expand bound, 4 edges per grid
 *    thread);
 *  - contract-expand and hybrid: full-grid contract-expand levels of at
 *    most grid_frontier queued entries, and at most one per grid thread,
 *    without chunked lists run a latency-first level body (one element per
 *    thread, short lists copied by their own thread, one queue reservation
 *    per CTA) instead of the tiled one (grid_frontier = 0: never;
 *    expand-contract and two-phase ignore it).
 * Both are off by default.  Results are the same either way.  No counterpart
 * in the reference. */
int b40c_enactor_set_narrow_levels(b40c_enactor_t *enactor, int team_ctas, int max_frontier,
                                   int grid_frontier);
/* The cluster size narrow levels run on for depth-label searches with the
 * enactor's current policy (0: off, or no cluster of that size fits). */
int b40c_enactor_narrow_team(b40c_enactor_t *enactor, int *team);

/* ---- host CSR graph builders (b40c/graph/builder/*.cuh, csr_graph.cuh) ---- */
typedef struct b40c_csr {
    int64_t nodes;
    int64_t edges;
    int *row_offsets;     /* nodes + 1 */
    int *column_indices;  /* edges */
} b40c_csr_t;
/* BuildGrid2dGraph (builder/grid2d.cuh:53-114): 4-neighbour lattice; the
 * reference appends one self-loop per vertex, kept here only if self_loops. */
int b40c_graph_grid2d(int width, int self_loops, b40c_csr_t *out);
/* BuildGrid3dGraph (builder/grid3d.cuh:53-129): 6-neighbour lattice. */
int b40c_graph_grid3d(int width, int self_loops, b40c_csr_t *out);
/* Graph500-style R-MAT (cf. BuildRmatGraph, builder/rmat.cuh:127-206):
 * 2^scale vertices, edge_factor * 2^scale generated edges with quadrant
 * probabilities a, b, c (d = 1-a-b-c), counter-based RNG from seed; self-loops
 * dropped; undirected adds the reverse of every edge; duplicates kept; rows
 * keep generation order. */
int b40c_graph_rmat(int scale, int edge_factor, double a, double b, double c,
                    uint64_t seed, int undirected, b40c_csr_t *out);
/* Erdos-Renyi G(n, p), undirected, no self-loops or duplicate edges. */
int b40c_graph_erdos_renyi(int nodes, double p, uint64_t seed, b40c_csr_t *out);
/* CsrGraph::FromCoo (csr_graph.cuh:108-152): stable sort by row. */
int b40c_graph_from_coo(int nodes, int64_t num_edges, const int *rows,
                        const int *cols, b40c_csr_t *out);
/* Graph files (b40c/graph/builder/market.cuh, metis.cuh, dimacs.cuh; the
 * BuildMarketGraph / BuildMetisGraph / BuildDimacsGraph readers used by
 * test/bfs/test_bfs.cu:981-1036).  Matrix Market entry "a b" is the edge
 * b-1 -> a-1 as the reference reads it; undirected adds each reverse edge. */
int b40c_graph_read_market(const char *path, int undirected, b40c_csr_t *out);
int b40c_graph_read_metis(const char *path, b40c_csr_t *out);
int b40c_graph_read_dimacs(const char *path, int undirected, b40c_csr_t *out);
/* Frees the arrays of a b40c_csr_t filled by this library. */
int b40c_csr_free(b40c_csr_t *csr);
/* num_sources vertex ids drawn uniformly (with a seeded RNG) among vertices of degree > 0. */
int b40c_graph_sample_sources(const b40c_csr_t *csr, int num_sources, uint64_t seed, int *sources);

/* ---- batched searches (no reference counterpart: the reference runs one
 * search per EnactSearch) -------------------------------------------------
 * Many (graph, source) searches over resident graphs run in one persistent
 * launch (expand-contract); each search has its own labels.  A batch can be
 * captured into a CUDA graph and replayed when run again unchanged. */
typedef struct b40c_batch b40c_batch_t;
int b40c_batch_create(int mark_predecessors, b40c_batch_t **out);
int b40c_batch_destroy(b40c_batch_t *batch);
/* Uploads a graph (validated like FromHostProblem); *graph_id names it. */
int b40c_batch_add_graph(b40c_batch_t *batch, int nodes, int edges, const int *h_column_indices,
                         const int *h_row_offsets, int *graph_id);
/* Same knobs as b40c_enactor_set_policy (expand-contract defaults). */
int b40c_batch_set_policy(b40c_batch_t *batch, int cta_threads, int warp_gather_threshold,
                          int cta_gather_threshold, int cull_flags);
int b40c_batch_set_stream(b40c_batch_t *batch, void *stream);
/* Bottom-up levels per search, as b40c_enactor_set_direction_optimizing
 * (default alpha = 14, beta = 24; alpha = 0: top-down only): a search over a
 * symmetric graph switches direction by its own frontier, independently of
 * the other searches of the batch.  Depth labels only. */
int b40c_batch_set_direction_optimizing(b40c_batch_t *batch, int alpha, int beta);
/* Runs search i from sources[i] on graph graph_ids[i], i < num_searches, and
 * waits.  use_cuda_graph captures the launch sequence (pool clears, admission
 * kernel, persistent kernel) once and replays it for identical batches. */
int b40c_batch_run(b40c_batch_t *batch, int num_searches, const int *graph_ids, const int *sources,
                   int use_cuda_graph);
int b40c_batch_run_async(b40c_batch_t *batch, int num_searches, const int *graph_ids,
                         const int *sources, int use_cuda_graph);
int b40c_batch_sync(b40c_batch_t *batch);
/* Labels of search i of the last batch (its graph's node count entries). */
int b40c_batch_extract(b40c_batch_t *batch, int search, int *h_labels);
/* search_depth of search i as the expand-contract enactor reports it. */
int b40c_batch_search_depth(b40c_batch_t *batch, int search, int *depth);
/* Device time of the last batch, CUDA events around its launch sequence. */
int b40c_batch_last_elapsed_ms(b40c_batch_t *batch, float *ms);

/* ---- serving (no reference counterpart) ----------------------------------
 * BFS queries over resident graphs with continuous batching: queries are
 * admitted into up to max_slots concurrent searches while the HBM budget's
 * label, mask, frontier and chunk pools allow, run together in epochs of the
 * persistent multi-search kernel, and retire as they finish, freeing room
 * for the queries that arrived meanwhile. */
typedef struct b40c_server b40c_server_t;
int b40c_server_create(int mark_predecessors, int max_slots, long long hbm_budget_bytes, b40c_server_t **out);
int b40c_server_destroy(b40c_server_t *server);
int b40c_server_add_graph(b40c_server_t *server, int nodes, int edges, const int *h_column_indices,
                          const int *h_row_offsets, int *graph_id);
/* Bottom-up levels per query, as b40c_batch_set_direction_optimizing. */
int b40c_server_set_direction_optimizing(b40c_server_t *server, int alpha, int beta);
/* Policy as b40c_batch_set_policy, plus the level cap of one epoch (0 keeps). */
int b40c_server_set_policy(b40c_server_t *server, int cta_threads, int warp_gather_threshold,
                           int cta_gather_threshold, int cull_flags, int epoch_levels);
/* Replays a trace in real time: query i (graph_ids[i], sources[i]) arrives
 * arrival_us[i] microseconds after the call (non-decreasing).  Returns when
 * every query finished; latency_us[i] = completion - arrival on the host
 * clock; labels_out[i], when labels_out and it are non-NULL, receives query
 * i's labels; *makespan_us (may be NULL) the time of the last completion. */
int b40c_server_run_trace(b40c_server_t *server, int n, const int *graph_ids, const int *sources,
                          const double *arrival_us, double *latency_us, int **labels_out, double *makespan_us);
/* Epochs run and the largest number of concurrent searches in the last trace. */
int b40c_server_stats(b40c_server_t *server, long long *epochs, long long *max_active);

/* ---- search without allocation (no counterpart in the reference) --------
 * For callers that must not allocate device memory while they search:
 * frameworks whose allocator owns all device memory, and latency-bound loops
 * that cannot afford the synchronisation cudaMalloc/cudaFree may cause.  Runs
 * one fused
 * expand-contract search (default policy, depth labels) over a CSR the caller
 * already holds on the current device: d_row_offsets (nodes + 1 entries,
 * non-decreasing from 0 to edges) and d_column_indices (edges entries, each
 * in [0, nodes)), writing nodes depth labels to d_labels (-1 = unreached).
 * *search_depth (may be NULL) gets the value b40c_enactor_get_statistics
 * reports for that search.  Synchronous on stream (NULL = default stream).
 * Allocates nothing: its scratch memory (counters, visited bitmask, frontier
 * queues, chunk tables) comes from one static 32 MiB device array that every
 * GPU loading the library holds until exit; a graph whose scratch would not
 * fit (about 1M vertices with 16M edges fits) is rejected with
 * B40C_ERR_INVALID_VALUE and a message naming both sizes.  The first call in
 * each device's CUDA context looks up that array's device address; make it
 * before any stream capture.  All calls on a device share the array: calls
 * that overlap on the GPU race and corrupt each other's results. */
int b40c_enact_search_no_alloc(int nodes, int edges, const int *d_row_offsets,
                               const int *d_column_indices, int src, int *d_labels,
                               int *search_depth, void *stream);

/* ---- failure detection -------------------------------------------------- */
/* Runs the bounded grid barrier on a cooperative grid with one arrival that
 * never comes: every block gives up after wait_limit_us and the call returns
 * B40C_ERR_LAUNCH_TIMEOUT with the context still usable. */
int b40c_debug_barrier_timeout(int grid_size, long long wait_limit_us);

#ifdef __cplusplus
}
#endif
#endif /* B40C_BFS_H */
