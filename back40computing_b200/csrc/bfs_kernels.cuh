// Launch interface between the host orchestration (bfs_host.cu) and the
// sm_100a BFS kernels (bfs_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "bfs_device.cuh"

namespace b40c_b200 {

enum Strategy : int {
    STRATEGY_EXPAND_CONTRACT = 0,
    STRATEGY_CONTRACT_EXPAND = 1,
    STRATEGY_TWO_PHASE = 2,
    STRATEGY_HYBRID = 3,  // contract-expand or two-phase per level, by frontier size (fused only)
};

enum CullFlags : unsigned {
    CULL_WARP = 1u,     // __match_any_sync duplicate cull inside a warp
    CULL_HISTORY = 2u,  // per-CTA shared-memory history cache of visited-mask words
};

// One record per BFS level (per phase for two-phase), written by one thread
// of the kernel that runs it: %globaltimer at its start, the input frontier
// queue length and the numbers of CTA and warp chunks it takes as input.
struct LevelRecord {
    unsigned long long t_start;
    unsigned frontier;
    unsigned chunks;
    unsigned wchunks;
    unsigned bottom_up;  // 1 when the level ran bottom-up (direction-optimizing)
    unsigned long long t_work_end = 0;  // when the last CTA finished the level's work (before its barrier)
};

// Everything a BFS kernel needs, passed by value.
struct BfsParams {
    const int *row_offsets;  // nodes + 1
    const int *col;          // edges (+4 padding entries for 16-byte tail loads)
    int *labels;             // nodes: depth, or predecessor when mark_pred
    unsigned *mask;          // visited bitmask, bit (v & 31) of word v >> 5
    unsigned *mask_snap;     // predecessor labels, bottom-up levels: copy of mask at the level's start
    int *queue[2];           // frontier ping-pong
    int *pred_queue[2];      // predecessor ping-pong (edge frontiers, mark_pred)
    int4 *chunks[2];         // CTA chunks of neighbour lists, ping-pong by phase: {start, len, pred, 0}
    int4 *wchunks[2];        // warp chunks of neighbour lists, same layout
    LevelRecord *levels;     // per-level log (level_cap records)
    Counters *ctr;
    unsigned long long wait_ns;      // grid-barrier spin limit
    unsigned long long cond_handle;  // cudaGraphConditionalHandle (per-level graphs)
    long long qcap;                  // elements per frontier queue
    int chunk_cap;                   // entries of each CTA chunk table
    int wchunk_cap;                  // entries of each warp chunk table
    int level_cap;                   // entries of levels
    int vec_end;                     // 16-byte loads of col are safe below this index
    int nodes;
    int src;
    int warp_th;  // lists >= warp_th are cut into warp chunks; shorter ones go through a warp scan
    int cta_th;   // lists >= cta_th are cut into CTA chunks
    unsigned cull_flags;
    // Direction-optimizing expand-contract (fused only; the graph must be
    // symmetric): a level runs bottom-up once the frontier's edges exceed the
    // unvisited vertices' edges / do_alpha, and returns to top-down once the
    // frontier holds fewer than nodes / do_beta vertices and shrinks.
    // do_alpha = 0: top-down only.
    unsigned do_alpha;
    unsigned do_beta;
    long long edges;  // CSR entries (for the unvisited-edge count)
    // Bottom-up levels: per vertex, its neighbour of highest degree as
    // (degree << 32) | id (0: no neighbours); probed before the list is read.
    const unsigned long long *heavy;
    // INSTRUMENT: per CTA of a fused kernel, the %globaltimer ns it spent in
    // level work (barrier waits excluded), written at the kernel's end; NULL: off.
    unsigned long long *cta_busy;
    // 1: stream the column array through L2 with evict_first (it is large
    // next to L2); 0: ordinary caching (the graph fits in L2).
    int stream_col;
    // 1: bottom-up steps stage their row offsets, heaviest-neighbour keys and
    // mask words in shared memory with bulk copies, one step ahead; the
    // arrays then carry ROW_PAD / HEAVY_PAD / MASK_PAD_BYTES of padding.
    int stage_bu;
    // 1: count every phase's raw edge frontier (INSTRUMENT's total_queued);
    // 0: only phases that cull while they gather count it (their queue
    // alone would stop the level loop early).
    int count_raw;
    // Narrow launch (one thread-block cluster): it runs levels while their
    // input is an edge-frontier queue of at most narrow_max entries with no
    // chunked lists, and leaves the rest to the full-grid launch after it.
    unsigned narrow_max;
    // Full-grid levels of at most flat_max queued edges without chunked lists
    // run contract-expand's latency-first body (ce_flat_level); 0: never.
    unsigned flat_max;
};

// Padding of the device arrays a staged bottom-up step copies in whole
// 16-byte units past their ends.
constexpr int ROW_PAD = 4;          // int entries after row_offsets[nodes]
constexpr int HEAVY_PAD = 2;        // keys after heavy[nodes - 1]
constexpr int MASK_PAD_BYTES = 16;  // bytes after the last visited-mask word

// Edges per CTA chunk: four passes of one 16-byte load per thread of a CTA.
template <int THREADS>
__host__ __device__ constexpr int chunk_edges() { return THREADS * 16; }
// Edges per warp chunk: four passes of one 16-byte load per lane.
constexpr int WARP_CHUNK = 512;

struct KernelConfig {
    int strategy;
    int threads;  // 128, 256 or 512
    bool mark_pred;
    bool stage_bu = false;  // the launch carries the bottom-up stage buffers (BfsParams::stage_bu)
};

// Enqueues the per-search initialisation (counters, source) on stream.
cudaError_t launch_search_init(const BfsParams &p, const KernelConfig &kc, cudaStream_t stream);
// Largest co-resident grid of the fused kernel (SMs x occupancy).
cudaError_t fused_grid_limit(const KernelConfig &kc, int *grid);
// Grid of the per-level kernels (SMs x occupancy).
cudaError_t level_grid_limit(const KernelConfig &kc, int *grid);
// Two 64-bit hash sums over the CSR's entries, of (u, v) and of (v, u); equal
// sums mean the graph is symmetric (up to a hash collision).  sums[0..3] must
// start at zero.
cudaError_t launch_symmetry_hash(const int *row_offsets, const int *col, int nodes, long long edges,
                                 unsigned long long *sums, cudaStream_t stream);
// Per vertex v, the neighbour u of highest degree as (deg(u) << 32) | u (the
// largest key, so ties go to the larger id); 0 for a vertex without
// neighbours.  keys[0..nodes) must start at zero.
cudaError_t launch_heavy_neighbour(const int *row_offsets, const int *col, int nodes, long long edges,
                                   unsigned long long *keys, cudaStream_t stream);
// Reset's state initialisation in one launch: labels[0..nodes) := -1 (labels
// 16-byte aligned), mask[0..mask_words) := 0.
cudaError_t launch_reset_state(int *labels, long long nodes, unsigned *mask, long long mask_words,
                               cudaStream_t stream);
// CSR validity on the device: out[0] = first row whose offsets decrease,
// out[1] = first column entry outside [0, nodes); ~0 when none.  out[0..1]
// must start at ~0.
cudaError_t launch_csr_check(const int *row_offsets, const int *col, int nodes, long long edges,
                             unsigned long long *out, cudaStream_t stream);
// Cooperative launch of the persistent kernel that runs every BFS level.
cudaError_t launch_fused(const BfsParams &p, const KernelConfig &kc, int grid, cudaStream_t stream);
// Whether strategy kc.strategy has a narrow kernel (the levels of small
// frontiers on one thread-block cluster), and the largest cluster of at most
// `want` CTAs it can launch (*team, 0 when none fits or there is no kernel).
cudaError_t narrow_team_limit(const KernelConfig &kc, int want, int *team);
// The narrow launch: one cluster of `team` CTAs runs the search's levels from
// Counters::resume while their frontiers stay within p.narrow_max, then
// writes the next level to Counters::resume for launch_fused's kernel.
cudaError_t launch_narrow(const BfsParams &p, const KernelConfig &kc, int team, cudaStream_t stream);
// Builds a graph whose conditional-while node runs one BFS level per pass:
// level kernel(s), then a control kernel that advances the iteration and
// sets the loop condition on the device.  p.cond_handle is filled in.
cudaError_t build_level_graph(BfsParams &p, const KernelConfig &kc, int grid,
                              cudaGraphExec_t *exec, cudaGraph_t *graph);
// Debug/failure-detection probe: a cooperative grid whose barrier expects one
// more arrival than there are CTAs.  Returns the device error word.
cudaError_t run_barrier_timeout_probe(int grid, unsigned long long wait_ns, unsigned *error_out);

}  // namespace b40c_b200
