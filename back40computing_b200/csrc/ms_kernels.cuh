// Multi-search BFS: many searches, over many resident graphs, in one
// persistent launch.  Interface between ms_host.cu and ms_kernels.cu.
#pragma once

#include <cuda_runtime.h>

#include "bfs_kernels.cuh"

namespace b40c_b200 {

struct MsGraph {
    const int *row;  // nodes + 1
    const int *col;  // edges (+4 padding)
    int nodes;
    int vec_end;     // 16-byte column loads are safe below this index
    int edges;
    int symmetric;   // 1: every entry has its reverse (bottom-up levels allowed)
    // symmetric graphs: per vertex, its neighbour of highest degree as
    // (degree << 32) | id (0: none), probed by bottom-up levels first
    const unsigned long long *heavy;
};

// Direction-optimizing state of one search slot, updated at the start of
// every level by the bookkeeping CTA.
struct MsDir {
    unsigned long long explored;  // degrees summed over the slot's visited vertices
    unsigned visited;             // the slot's visited vertices
    unsigned prev_nf;             // its frontier size at the previous level
    int bottom_up;                // 1: the current level runs bottom-up
    int nodes;                    // the slot's graph, copied at admission so that the
    int edges;                    //   per-level decision reads nothing but this record
    int symmetric;                //   and the slot's counts
};

struct MsSlot {
    long long label_off;  // labels of this search start at labels + label_off
    long long mask_off;   // visited mask words start at mask + mask_off
    int graph;            // index into the graph table
    int start_level;      // level at which the search was admitted
    int nodes;            // nodes of its graph
    int pad;
};

// Per-slot progress written by the kernel.
struct MsSlotState {
    int active;        // 1 while the search runs
    int done_levels;   // EC iteration count at completion (search_depth + 1), -1 while running
    unsigned long long done_ns;  // %globaltimer when the search finished
};

struct MsParams {
    const MsGraph *graphs;
    const MsSlot *slots;
    MsSlotState *state;
    unsigned char *alive;     // [4][nslots]: alive[q&3][s] = search s has input for level q
    int nslots;
    int *labels;
    unsigned *mask;
    int2 *queue[2];           // frontier entries (slot, vertex)
    long long qcap;
    int4 *chunks[2];          // CTA chunks {start, len, pred, slot}
    int4 *wchunks[2];         // warp chunks, same layout
    int chunk_cap;
    int wchunk_cap;
    Counters *ctr;
    LevelRecord *levels;
    int level_cap;
    unsigned long long wait_ns;
    int warp_th;
    int cta_th;
    unsigned cull_flags;
    int max_levels;  // levels to run in this launch before returning (<= 0: until no work)
    int stop_on_retire;  // return at the level after one where a search retired
    // Direction-optimizing searches (do_alpha = 0: top-down only): per slot,
    // the vertices discovered as input of level q (nf) and their degree sum
    // (mf) at [(q & 3) * nslots + slot]; the direction state after level q at
    // [(q & 1) * nslots + slot]; the current
    // level's bottom-up flag; and bu_prefix[s] = the bottom-up steps (4 mask
    // words each) of the slots before s, bu_prefix[nslots] their total.
    unsigned do_alpha;
    unsigned do_beta;
    unsigned *nf;
    unsigned long long *mf;
    MsDir *dir;
    unsigned char *bu;
    unsigned *bu_prefix;
};

struct MsKernelConfig {
    int threads;  // 128, 256, 512
    bool mark_pred;
};

// Whether a resident graph is symmetric (the hash check of
// launch_symmetry_hash; allocates and frees a 32-byte buffer, waits).
cudaError_t ms_graph_symmetric(const int *d_row, const int *d_col, int nodes, long long edges, int *symmetric);
// Allocates and fills the heaviest-neighbour keys of a resident graph
// (launch_heavy_neighbour), waiting for them; *keys = nullptr when nodes == 0.
cudaError_t ms_graph_heavy(const int *d_row, const int *d_col, int nodes, long long edges, unsigned long long **keys);
// Largest co-resident grid of the multi-search kernel.
cudaError_t ms_grid_limit(const MsKernelConfig &kc, int *grid);
// Cooperative launch: runs levels from Counters::cur_it until no search has
// work or max_levels levels ran; leaves the ring ready to continue.
cudaError_t ms_launch(const MsParams &p, const MsKernelConfig &kc, int grid, cudaStream_t stream);
// Clears labels (to -1) and visited-mask words (to 0) of the given slots.
cudaError_t ms_clear_slots(const MsParams &p, const int *d_slots, int count, cudaStream_t stream);
// Admits searches: for each (slot, source) pair labels and marks the source
// and places its list as input of level Counters::cur_it.  The slots' labels
// and masks must be cleared beforehand.
cudaError_t ms_admit(const MsParams &p, const MsKernelConfig &kc, const int2 *d_slot_src, int count,
                     cudaStream_t stream);

}  // namespace b40c_b200
