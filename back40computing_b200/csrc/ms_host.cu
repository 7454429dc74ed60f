// Host side of the multi-search BFS: batched searches (b40c_batch_*) over a
// set of resident graphs, run as one persistent launch per batch and
// optionally captured into a CUDA graph that later batches replay.
//
// Device layout of a batch of S searches: one labels pool (sum of the
// searches' vertex counts), one visited-mask pool (32-bit words, one span per
// search), a frontier of (slot, vertex) pairs sized for every vertex of every
// search, and two chunk tables sized for every search's edges.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "b40c_bfs.h"
#include "host_common.h"
#include "ms_kernels.cuh"

using namespace b40c_b200;

namespace {

int cuda_fail(cudaError_t e, const char *what) {
    return set_error(int(e), "%s failed (CUDA error %d: %s)", what, int(e), cudaGetErrorString(e));
}
#define CUDA_TRY(call, what)                                 \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) return cuda_fail(_e, what);   \
    } while (0)

template <class T>
int grow(T **ptr, size_t *cap, size_t need, const char *what) {
    if (*cap >= need && *ptr) return B40C_SUCCESS;
    cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    CUDA_TRY(cudaMalloc(ptr, sizeof(T) * std::max<size_t>(need, 1)), what);
    *cap = need;
    return B40C_SUCCESS;
}

struct GraphRes {
    int *d_row = nullptr;
    int *d_col = nullptr;
    int nodes = 0;
    long long edges = 0;
    int symmetric = 0;
    unsigned long long *d_heavy = nullptr;  // symmetric graphs: heaviest neighbour per vertex
};

}  // namespace

struct b40c_batch {
    int device = 0;
    bool mark_pred = false;
    int threads = 512, warp_th = 128, cta_th = 1024;  // 512-thread CTAs: measured best for the mixed batch
    unsigned cull_flags = CULL_HISTORY;
    unsigned do_alpha = 14, do_beta = 24;  // direction-optimizing (published alpha, beta); 0: top-down only
    unsigned long long wait_ns = 5000000000ull;
    std::vector<GraphRes> graphs;
    MsGraph *d_graphs = nullptr;
    size_t graphs_cap = 0;
    // per-batch buffers
    int nslots = 0;
    std::vector<long long> label_off;
    std::vector<int> slot_nodes;
    MsSlot *d_slots = nullptr;
    size_t slots_cap = 0;
    MsSlotState *d_state = nullptr;
    size_t state_cap = 0;
    unsigned char *d_alive = nullptr;
    size_t alive_cap = 0;
    int *d_labels = nullptr;
    size_t labels_cap = 0;
    unsigned *d_mask = nullptr;
    size_t mask_cap = 0;
    int2 *d_queue[2] = {nullptr, nullptr};
    size_t queue_cap[2] = {0, 0};
    int4 *d_chunks[2] = {nullptr, nullptr};
    size_t chunk_cap[2] = {0, 0};
    int4 *d_wchunks[2] = {nullptr, nullptr};
    size_t wchunk_cap[2] = {0, 0};
    int2 *d_admit = nullptr;
    size_t admit_cap = 0;
    unsigned *d_nf = nullptr;  // direction-optimizing state, per slot
    size_t nf_cap = 0;
    unsigned long long *d_mf = nullptr;
    size_t mf_cap = 0;
    MsDir *d_dir = nullptr;
    size_t dir_cap = 0;
    unsigned char *d_bu = nullptr;
    size_t bu_cap = 0;
    unsigned *d_bu_prefix = nullptr;
    size_t bu_prefix_cap = 0;
    Counters *d_ctr = nullptr;
    Counters *h_ctr = nullptr;
    MsSlotState *h_state = nullptr;  // pinned
    size_t h_state_cap = 0;
    MsSlot *h_slots = nullptr;  // pinned staging
    int2 *h_admit = nullptr;    // pinned staging
    size_t h_stage_cap = 0;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    bool pending = false;
    // captured launch sequence
    cudaGraphExec_t exec = nullptr;
    std::vector<int> exec_key;
    MsParams params{};
    int grid = 0;
};

namespace {

cudaStream_t bstream(b40c_batch *b) { return b->stream ? b->stream : b->own_stream; }

int ensure_staging(b40c_batch *b, size_t n) {
    if (b->h_stage_cap >= n && b->h_slots) return B40C_SUCCESS;
    cudaFreeHost(b->h_slots);
    cudaFreeHost(b->h_admit);
    cudaFreeHost(b->h_state);
    b->h_slots = nullptr;
    b->h_admit = nullptr;
    b->h_state = nullptr;
    b->h_stage_cap = 0;
    CUDA_TRY(cudaHostAlloc(&b->h_slots, sizeof(MsSlot) * n, cudaHostAllocDefault), "batch pinned slots");
    CUDA_TRY(cudaHostAlloc(&b->h_admit, sizeof(int2) * n, cudaHostAllocDefault), "batch pinned sources");
    CUDA_TRY(cudaHostAlloc(&b->h_state, sizeof(MsSlotState) * n, cudaHostAllocDefault), "batch pinned states");
    b->h_stage_cap = n;
    return B40C_SUCCESS;
}

// Enqueues one batch: clear the pools, admit every search at level 0, run the
// persistent kernel until no search has work.
int enqueue_batch(b40c_batch *b, size_t labels_total, size_t mask_total, cudaStream_t s) {
    CUDA_TRY(cudaMemsetAsync(b->d_labels, 0xff, sizeof(int) * labels_total, s), "labels clear");
    CUDA_TRY(cudaMemsetAsync(b->d_mask, 0, sizeof(unsigned) * mask_total, s), "mask clear");
    CUDA_TRY(cudaMemsetAsync(b->d_alive, 0, 4 * size_t(b->nslots), s), "alive clear");
    CUDA_TRY(cudaMemsetAsync(b->d_ctr, 0, offsetof(Counters, sticky), s), "counters clear");
    CUDA_TRY(cudaMemcpyAsync(b->d_slots, b->h_slots, sizeof(MsSlot) * b->nslots, cudaMemcpyHostToDevice, s),
             "slot table upload");
    CUDA_TRY(cudaMemcpyAsync(b->d_admit, b->h_admit, sizeof(int2) * b->nslots, cudaMemcpyHostToDevice, s),
             "source upload");
    MsKernelConfig kc{b->threads, b->mark_pred};
    CUDA_TRY(ms_admit(b->params, kc, b->d_admit, b->nslots, s), "admission kernel");
    CUDA_TRY(ms_launch(b->params, kc, b->grid, s), "multi-search kernel launch");
    return B40C_SUCCESS;
}

int finish_batch(b40c_batch *b) {
    cudaStream_t s = bstream(b);
    CUDA_TRY(cudaMemcpyAsync(b->h_ctr, b->d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s), "counters copy");
    CUDA_TRY(cudaMemcpyAsync(b->h_state, b->d_state, sizeof(MsSlotState) * b->nslots, cudaMemcpyDeviceToHost, s),
             "state copy");
    CUDA_TRY(cudaStreamSynchronize(s), "batched BFS");
    if (b->pending) {
        cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
        b->pending = false;
    }
    unsigned err = b->h_ctr->sticky | b->h_ctr->error;
    if (err) {
        cudaMemsetAsync(&b->d_ctr->sticky, 0, sizeof(unsigned), s);
        cudaStreamSynchronize(s);
        if (err & ERR_BAD_VERTEX) return set_error(B40C_ERR_INVALID_VALUE, "batch: vertex id out of range");
        if (err & ERR_BARRIER_TIMEOUT) return set_error(B40C_ERR_LAUNCH_TIMEOUT, "batch: grid barrier wait timed out");
        if (err & ERR_OVERFLOW) return set_error(B40C_ERR_INVALID_CONFIGURATION, "batch: frontier queue overflow");
        return set_error(B40C_ERR_LAUNCH_TIMEOUT, "batch: level loop limit");
    }
    return B40C_SUCCESS;
}

}  // namespace

extern "C" int b40c_batch_create(int mark_predecessors, b40c_batch_t **out) {
    clear_error();
    if (!out) return set_error(B40C_ERR_INVALID_VALUE, "NULL out");
    b40c_batch *b = new (std::nothrow) b40c_batch();
    if (!b) return set_error(B40C_ERR_MEMORY_ALLOCATION, "batch allocation");
    b->mark_pred = mark_predecessors != 0;
    cudaError_t e = cudaGetDevice(&b->device);
    if (!e) e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
    if (!e) e = cudaEventCreate(&b->ev0);
    if (!e) e = cudaEventCreate(&b->ev1);
    if (!e) e = cudaMalloc(&b->d_ctr, sizeof(Counters));
    if (!e) e = cudaMemset(b->d_ctr, 0, sizeof(Counters));
    if (!e) e = cudaHostAlloc(&b->h_ctr, sizeof(Counters), cudaHostAllocDefault);
    if (e) {
        delete b;
        return cuda_fail(e, "batch creation");
    }
    *out = b;
    return B40C_SUCCESS;
}

extern "C" int b40c_batch_destroy(b40c_batch_t *b) {
    clear_error();
    if (!b) return B40C_SUCCESS;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(bstream(b));
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (auto &g : b->graphs) {
        cudaFree(g.d_row);
        cudaFree(g.d_col);
        cudaFree(g.d_heavy);
    }
    cudaFree(b->d_graphs);
    cudaFree(b->d_slots);
    cudaFree(b->d_state);
    cudaFree(b->d_alive);
    cudaFree(b->d_labels);
    cudaFree(b->d_mask);
    for (int i = 0; i < 2; i++) {
        cudaFree(b->d_queue[i]);
        cudaFree(b->d_chunks[i]);
        cudaFree(b->d_wchunks[i]);
    }
    cudaFree(b->d_admit);
    cudaFree(b->d_nf);
    cudaFree(b->d_mf);
    cudaFree(b->d_dir);
    cudaFree(b->d_bu);
    cudaFree(b->d_bu_prefix);
    cudaFree(b->d_ctr);
    cudaFreeHost(b->h_ctr);
    cudaFreeHost(b->h_state);
    cudaFreeHost(b->h_slots);
    cudaFreeHost(b->h_admit);
    cudaEventDestroy(b->ev0);
    cudaEventDestroy(b->ev1);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    delete b;
    return B40C_SUCCESS;
}

extern "C" int b40c_batch_add_graph(b40c_batch_t *b, int nodes, int edges, const int *h_col, const int *h_row,
                                    int *graph_id) {
    clear_error();
    if (!b || !graph_id || nodes <= 0 || edges < 0 || !h_row || (edges && !h_col))
        return set_error(B40C_ERR_INVALID_VALUE, "batch_add_graph: invalid arguments");
    if (h_row[0] != 0 || h_row[nodes] != edges)
        return set_error(B40C_ERR_INVALID_VALUE, "batch_add_graph: row offsets do not span [0, edges]");
    for (int v = 0; v < nodes; v++)
        if (h_row[v + 1] < h_row[v])
            return set_error(B40C_ERR_INVALID_VALUE, "batch_add_graph: row offsets decrease at %d", v);
    for (int k = 0; k < edges; k++)
        if ((unsigned)h_col[k] >= (unsigned)nodes)
            return set_error(B40C_ERR_INVALID_VALUE, "batch_add_graph: column index %d out of range", h_col[k]);
    CUDA_TRY(cudaSetDevice(b->device), "cudaSetDevice");
    GraphRes g;
    g.nodes = nodes;
    g.edges = edges;
    // Frees the graph's device arrays if a step below fails before the
    // batch owns them.
    struct Unwind {
        GraphRes *g;
        bool owned = false;
        ~Unwind() {
            if (owned) return;
            cudaFree(g->d_row);
            cudaFree(g->d_col);
            cudaFree(g->d_heavy);
        }
    } unwind{&g};
    CUDA_TRY(cudaMalloc(&g.d_row, sizeof(int) * (size_t(nodes) + 1)), "batch graph row offsets");
    CUDA_TRY(cudaMalloc(&g.d_col, sizeof(int) * (size_t(edges) + 4)), "batch graph column indices");
    CUDA_TRY(cudaMemcpy(g.d_row, h_row, sizeof(int) * (size_t(nodes) + 1), cudaMemcpyHostToDevice), "upload");
    CUDA_TRY(cudaMemset(g.d_col + edges, 0, 4 * sizeof(int)), "column padding");
    if (edges) CUDA_TRY(cudaMemcpy(g.d_col, h_col, sizeof(int) * size_t(edges), cudaMemcpyHostToDevice), "upload");
    CUDA_TRY(ms_graph_symmetric(g.d_row, g.d_col, nodes, edges, &g.symmetric), "graph symmetry check");
    if (g.symmetric)
        CUDA_TRY(ms_graph_heavy(g.d_row, g.d_col, nodes, edges, &g.d_heavy), "heaviest-neighbour keys");
    // Refresh the device graph table with the new graph appended; the batch
    // owns the graph only once the table holds it, so that a failure here
    // leaves b->graphs and the device table as they were.
    std::vector<MsGraph> table(b->graphs.size() + 1);
    for (size_t i = 0; i < b->graphs.size(); i++)
        table[i] = MsGraph{b->graphs[i].d_row, b->graphs[i].d_col, b->graphs[i].nodes,
                           int(b->graphs[i].edges + 4), int(b->graphs[i].edges), b->graphs[i].symmetric,
                           b->graphs[i].d_heavy};
    table.back() = MsGraph{g.d_row, g.d_col, g.nodes, int(g.edges + 4), int(g.edges), g.symmetric, g.d_heavy};
    int rc = grow(&b->d_graphs, &b->graphs_cap, table.size(), "batch graph table");
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(b->d_graphs, table.data(), sizeof(MsGraph) * table.size(), cudaMemcpyHostToDevice),
             "graph table upload");
    b->graphs.push_back(g);
    unwind.owned = true;
    *graph_id = int(b->graphs.size()) - 1;
    return B40C_SUCCESS;
}

extern "C" int b40c_batch_set_direction_optimizing(b40c_batch_t *b, int alpha, int beta) {
    clear_error();
    if (!b || alpha < 0 || beta < 0 || (alpha > 0 && beta == 0))
        return set_error(B40C_ERR_INVALID_VALUE, "direction switch: alpha >= 0, and beta >= 1 when alpha > 0");
    b->do_alpha = unsigned(alpha);
    b->do_beta = unsigned(beta);
    return B40C_SUCCESS;
}

extern "C" int b40c_batch_set_policy(b40c_batch_t *b, int cta_threads, int warp_th, int cta_th, int cull_flags) {
    clear_error();
    if (!b) return set_error(B40C_ERR_INVALID_VALUE, "NULL batch");
    if (cta_threads && cta_threads != 128 && cta_threads != 256 && cta_threads != 512)
        return set_error(B40C_ERR_INVALID_VALUE, "cta_threads must be 128, 256 or 512");
    if (warp_th < 0 || cta_th < 0 || cull_flags < -1 || cull_flags > 3)
        return set_error(B40C_ERR_INVALID_VALUE, "invalid policy field");
    if (cta_threads) b->threads = cta_threads;
    if (warp_th) b->warp_th = warp_th;
    if (cta_th) b->cta_th = cta_th;
    if (cull_flags >= 0) b->cull_flags = unsigned(cull_flags);
    return B40C_SUCCESS;
}

extern "C" int b40c_batch_set_stream(b40c_batch_t *b, void *stream) {
    clear_error();
    if (!b) return set_error(B40C_ERR_INVALID_VALUE, "NULL batch");
    b->stream = (cudaStream_t)stream;
    return B40C_SUCCESS;
}

extern "C" int b40c_batch_run_async(b40c_batch_t *b, int num_searches, const int *graph_ids, const int *sources,
                                    int use_cuda_graph) {
    clear_error();
    if (!b || num_searches <= 0 || !graph_ids || !sources)
        return set_error(B40C_ERR_INVALID_VALUE, "batch_run: invalid arguments");
    for (int s = 0; s < num_searches; s++) {
        if (graph_ids[s] < 0 || graph_ids[s] >= (int)b->graphs.size())
            return set_error(B40C_ERR_INVALID_VALUE, "batch_run: search %d names graph %d of %zu", s, graph_ids[s],
                             b->graphs.size());
        if (sources[s] < 0 || sources[s] >= b->graphs[graph_ids[s]].nodes)
            return set_error(B40C_ERR_INVALID_VALUE, "batch_run: search %d source %d out of range", s, sources[s]);
    }
    CUDA_TRY(cudaSetDevice(b->device), "cudaSetDevice");
    cudaStream_t s = bstream(b);
    // Layout and capacities.
    const int CH_MIN = chunk_edges<128>();
    size_t labels_total = 0, mask_total = 0, chunks_need = 64, wchunks_need = 64;
    b->label_off.assign(num_searches, 0);
    b->slot_nodes.assign(num_searches, 0);
    int rc = ensure_staging(b, size_t(num_searches));
    if (rc) return rc;
    const long long ct = std::max(1, std::max(b->cta_th, b->warp_th)), wt = std::max(1, b->warp_th);
    for (int i = 0; i < num_searches; i++) {
        const GraphRes &g = b->graphs[graph_ids[i]];
        MsSlot d{};
        d.label_off = (long long)labels_total;
        d.mask_off = (long long)mask_total;
        d.graph = graph_ids[i];
        d.start_level = 0;
        d.nodes = g.nodes;
        b->h_slots[i] = d;
        b->h_admit[i] = make_int2(i, sources[i]);
        b->label_off[i] = (long long)labels_total;
        b->slot_nodes[i] = g.nodes;
        labels_total += size_t(g.nodes);
        mask_total += size_t((g.nodes + 31) / 32);
        chunks_need += size_t(g.edges / CH_MIN + 2 * (g.edges / ct) + 2);
        wchunks_need += size_t(g.edges / WARP_CHUNK + 2 * (g.edges / wt) + 2);
    }
    if (mask_total >= (size_t(1) << 32))
        return set_error(B40C_ERR_INVALID_VALUE, "batch_run: visited masks exceed 2^32 words");
    chunks_need = std::min<size_t>(chunks_need, size_t(1) << 30);
    wchunks_need = std::min<size_t>(wchunks_need, size_t(1) << 30);
    const bool grew = b->labels_cap < labels_total || b->mask_cap < mask_total || b->slots_cap < size_t(num_searches) ||
                      b->queue_cap[0] < labels_total + 1 || b->chunk_cap[0] < chunks_need ||
                      b->wchunk_cap[0] < wchunks_need;
    if ((rc = grow(&b->d_labels, &b->labels_cap, labels_total, "batch labels"))) return rc;
    if ((rc = grow(&b->d_mask, &b->mask_cap, mask_total, "batch visited masks"))) return rc;
    if ((rc = grow(&b->d_slots, &b->slots_cap, size_t(num_searches), "batch slot table"))) return rc;
    if ((rc = grow(&b->d_state, &b->state_cap, size_t(num_searches), "batch slot states"))) return rc;
    if ((rc = grow(&b->d_alive, &b->alive_cap, 4 * size_t(num_searches), "batch alive flags"))) return rc;
    if ((rc = grow(&b->d_admit, &b->admit_cap, size_t(num_searches), "batch sources"))) return rc;
    const size_t S = size_t(num_searches);
    if ((rc = grow(&b->d_nf, &b->nf_cap, 4 * S, "batch direction counts"))) return rc;
    if ((rc = grow(&b->d_mf, &b->mf_cap, 4 * S, "batch direction degree sums"))) return rc;
    if ((rc = grow(&b->d_dir, &b->dir_cap, 2 * S, "batch direction states"))) return rc;
    if ((rc = grow(&b->d_bu, &b->bu_cap, S, "batch bottom-up flags"))) return rc;
    if ((rc = grow(&b->d_bu_prefix, &b->bu_prefix_cap, S + 1, "batch bottom-up steps"))) return rc;
    for (int i = 0; i < 2; i++) {
        if ((rc = grow(&b->d_queue[i], &b->queue_cap[i], labels_total + 1, "batch frontier"))) return rc;
        if ((rc = grow(&b->d_chunks[i], &b->chunk_cap[i], chunks_need, "batch CTA chunks"))) return rc;
        if ((rc = grow(&b->d_wchunks[i], &b->wchunk_cap[i], wchunks_need, "batch warp chunks"))) return rc;
    }
    b->nslots = num_searches;
    MsKernelConfig kc{b->threads, b->mark_pred};
    int grid = 0;
    CUDA_TRY(ms_grid_limit(kc, &grid), "multi-search occupancy");
    MsParams p{};
    p.graphs = b->d_graphs;
    p.slots = b->d_slots;
    p.state = b->d_state;
    p.alive = b->d_alive;
    p.nslots = num_searches;
    p.labels = b->d_labels;
    p.mask = b->d_mask;
    p.queue[0] = b->d_queue[0];
    p.queue[1] = b->d_queue[1];
    p.qcap = (long long)std::min(b->queue_cap[0], b->queue_cap[1]);
    for (int i = 0; i < 2; i++) {
        p.chunks[i] = b->d_chunks[i];
        p.wchunks[i] = b->d_wchunks[i];
    }
    p.chunk_cap = int(std::min(b->chunk_cap[0], b->chunk_cap[1]));
    p.wchunk_cap = int(std::min(b->wchunk_cap[0], b->wchunk_cap[1]));
    p.ctr = b->d_ctr;
    p.wait_ns = b->wait_ns;
    p.warp_th = b->warp_th;
    p.cta_th = std::max(b->cta_th, b->warp_th);
    p.cull_flags = b->cull_flags;
    p.max_levels = 0;
    p.do_alpha = b->mark_pred ? 0u : b->do_alpha;
    p.do_beta = b->do_beta;
    p.nf = b->d_nf;
    p.mf = b->d_mf;
    p.dir = b->d_dir;
    p.bu = b->d_bu;
    p.bu_prefix = b->d_bu_prefix;
    const bool params_changed = grew || std::memcmp(&p, &b->params, sizeof(MsParams)) != 0 || grid != b->grid;
    b->params = p;
    b->grid = grid;

    CUDA_TRY(cudaEventRecord(b->ev0, s), "cudaEventRecord");
    if (use_cuda_graph) {
        std::vector<int> key(graph_ids, graph_ids + num_searches);
        key.insert(key.end(), sources, sources + num_searches);
        if (!b->exec || params_changed || key != b->exec_key) {
            if (b->exec) cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
            cudaStream_t cap = nullptr;
            CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream");
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            int erc = e ? cuda_fail(e, "cudaStreamBeginCapture") : enqueue_batch(b, labels_total, mask_total, cap);
            cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
            if (!erc && e2) erc = cuda_fail(e2, "cudaStreamEndCapture");
            if (!erc) {
                e = cudaGraphInstantiate(&b->exec, graph, 0);
                if (e) erc = cuda_fail(e, "cudaGraphInstantiate (batch)");
            }
            if (graph) cudaGraphDestroy(graph);
            cudaStreamDestroy(cap);
            if (erc) return erc;
            b->exec_key = key;
        }
        CUDA_TRY(cudaGraphLaunch(b->exec, s), "cudaGraphLaunch (batch)");
    } else {
        if ((rc = enqueue_batch(b, labels_total, mask_total, s))) return rc;
    }
    CUDA_TRY(cudaEventRecord(b->ev1, s), "cudaEventRecord");
    b->pending = true;
    return B40C_SUCCESS;
}

extern "C" int b40c_batch_sync(b40c_batch_t *b) {
    clear_error();
    if (!b) return set_error(B40C_ERR_INVALID_VALUE, "NULL batch");
    return finish_batch(b);
}

extern "C" int b40c_batch_run(b40c_batch_t *b, int num_searches, const int *graph_ids, const int *sources,
                              int use_cuda_graph) {
    int rc = b40c_batch_run_async(b, num_searches, graph_ids, sources, use_cuda_graph);
    if (rc) return rc;
    return finish_batch(b);
}

extern "C" int b40c_batch_extract(b40c_batch_t *b, int search, int *h_labels) {
    clear_error();
    if (!b || !h_labels || search < 0 || search >= b->nslots)
        return set_error(B40C_ERR_INVALID_VALUE, "batch_extract: invalid arguments");
    CUDA_TRY(cudaMemcpyAsync(h_labels, b->d_labels + b->label_off[search], sizeof(int) * size_t(b->slot_nodes[search]),
                             cudaMemcpyDeviceToHost, bstream(b)),
             "batch label copy");
    CUDA_TRY(cudaStreamSynchronize(bstream(b)), "batch label copy");
    return B40C_SUCCESS;
}

extern "C" int b40c_batch_search_depth(b40c_batch_t *b, int search, int *depth) {
    clear_error();
    if (!b || !depth || search < 0 || search >= b->nslots)
        return set_error(B40C_ERR_INVALID_VALUE, "batch_search_depth: invalid arguments");
    *depth = b->h_state[search].done_levels - 1;
    return B40C_SUCCESS;
}

extern "C" int b40c_batch_last_elapsed_ms(b40c_batch_t *b, float *ms) {
    clear_error();
    if (!b || !ms) return set_error(B40C_ERR_INVALID_VALUE, "NULL argument");
    *ms = b->last_ms;
    return B40C_SUCCESS;
}
