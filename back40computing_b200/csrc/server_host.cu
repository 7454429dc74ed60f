// Serving loop for BFS queries over resident graphs with continuous batching.
//
// b40c_server keeps graphs on the device and answers (graph, source) queries.
// Queries are admitted into search slots of the multi-search kernel while
// slots and HBM (a fixed budget split into label, mask, frontier and chunk
// pools) allow; admitted searches run together in epochs of the persistent
// kernel; an epoch ends a level after some search finishes (or after a level
// cap), the finished searches are retired and their memory returned, and the
// queries that arrived meanwhile are admitted before the next epoch.  A search
// keeps its labels and depth independent of what else runs beside it.
//
// b40c_server_run_trace replays a request trace in real time: query i arrives
// arrival_us[i] after the call starts, and its latency is completion time
// minus arrival time, measured on the host clock.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <thread>
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

// First-fit allocator over [0, capacity) with coalescing frees.
class RangePool {
  public:
    void reset(size_t capacity) {
        free_.clear();
        if (capacity) free_[0] = capacity;
        capacity_ = capacity;
    }
    bool alloc(size_t n, size_t *off) {
        if (n == 0) n = 1;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *off = it->first;
                size_t rest = it->second - n;
                size_t next = it->first + n;
                free_.erase(it);
                if (rest) free_[next] = rest;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t n) {
        if (n == 0) n = 1;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t capacity() const { return capacity_; }

  private:
    std::map<size_t, size_t> free_;
    size_t capacity_ = 0;
};

struct ResidentGraph {
    int *d_row = nullptr;
    int *d_col = nullptr;
    int nodes = 0;
    long long edges = 0;
    int symmetric = 0;
    unsigned long long *d_heavy = nullptr;  // symmetric graphs: heaviest neighbour per vertex
};

struct SlotUse {
    long long query = -1;
    size_t label_off = 0, mask_off = 0;
    size_t chunks = 0, wchunks = 0;
    int nodes = 0;
};

}  // namespace

struct b40c_server {
    int device = 0;
    bool mark_pred = false;
    int threads = 512, warp_th = 128, cta_th = 1024;  // 512-thread CTAs: measured best for the mixed batch
    unsigned cull_flags = CULL_HISTORY;
    unsigned long long wait_ns = 5000000000ull;
    int epoch_levels = 8;
    int max_slots = 0;
    std::vector<ResidentGraph> graphs;
    MsGraph *d_graphs = nullptr;
    // pools
    RangePool labels, masks;
    size_t chunk_cap = 0, wchunk_cap = 0, chunk_used = 0, wchunk_used = 0;
    MsSlot *d_slots = nullptr;
    MsSlotState *d_state = nullptr;
    unsigned char *d_alive = nullptr;
    int *d_labels = nullptr;
    unsigned *d_mask = nullptr;
    int2 *d_queue[2] = {nullptr, nullptr};
    int4 *d_chunks[2] = {nullptr, nullptr};
    int4 *d_wchunks[2] = {nullptr, nullptr};
    int2 *d_admit = nullptr;
    int *d_clear = nullptr;
    unsigned do_alpha = 14, do_beta = 24;  // direction-optimizing (published alpha, beta); 0: top-down only
    unsigned *d_nf = nullptr;              // direction-optimizing state, per slot
    unsigned long long *d_mf = nullptr;
    MsDir *d_dir = nullptr;
    unsigned char *d_bu = nullptr;
    unsigned *d_bu_prefix = nullptr;
    Counters *d_ctr = nullptr;
    Counters *h_ctr = nullptr;
    MsSlot *h_slots = nullptr;
    MsSlotState *h_state = nullptr;
    int2 *h_admit = nullptr;
    int *h_clear = nullptr;
    std::vector<SlotUse> use;
    std::vector<int> free_slots;
    cudaStream_t stream = nullptr;
    int grid = 0;
    MsParams params{};
    // statistics of the last trace
    long long epochs = 0, max_active = 0;
};

namespace {

int server_alloc(b40c_server *s, long long budget) {
    // Per vertex of label capacity: 4 B label + 16 B frontier (two (slot, v)
    // queues) + 1/8 B mask; chunk tables get a quarter of the budget.
    const double per_vertex = 4.0 + 16.0 + 0.125;
    const long long chunk_bytes = budget / 4;
    const size_t V = size_t(double(budget - chunk_bytes) / per_vertex);
    s->chunk_cap = size_t(chunk_bytes / 2 / 16 / 4);         // two CTA tables
    s->wchunk_cap = size_t(chunk_bytes / 2 / 16 / 4) * 3;    // two warp tables, three times as many
    s->chunk_cap = std::min<size_t>(s->chunk_cap, size_t(1) << 30);
    s->wchunk_cap = std::min<size_t>(s->wchunk_cap, size_t(1) << 30);
    const size_t W = (V + 31) / 32 + size_t(s->max_slots);  // mask words incl. per-slot rounding
    if (V < 1024 || W >= (size_t(1) << 32))
        return set_error(B40C_ERR_INVALID_VALUE, "server: HBM budget %lld bytes out of range", budget);
    s->labels.reset(V);
    s->masks.reset(W);
    const size_t S = size_t(s->max_slots);
    CUDA_TRY(cudaMalloc(&s->d_labels, sizeof(int) * V), "server labels pool");
    CUDA_TRY(cudaMalloc(&s->d_mask, sizeof(unsigned) * W), "server mask pool");
    for (int i = 0; i < 2; i++) {
        CUDA_TRY(cudaMalloc(&s->d_queue[i], sizeof(int2) * (V + 1)), "server frontier");
        CUDA_TRY(cudaMalloc(&s->d_chunks[i], sizeof(int4) * s->chunk_cap), "server CTA chunks");
        CUDA_TRY(cudaMalloc(&s->d_wchunks[i], sizeof(int4) * s->wchunk_cap), "server warp chunks");
    }
    CUDA_TRY(cudaMalloc(&s->d_slots, sizeof(MsSlot) * S), "server slot table");
    CUDA_TRY(cudaMalloc(&s->d_state, sizeof(MsSlotState) * S), "server slot states");
    CUDA_TRY(cudaMalloc(&s->d_alive, 4 * S), "server alive flags");
    CUDA_TRY(cudaMalloc(&s->d_admit, sizeof(int2) * S), "server admissions");
    CUDA_TRY(cudaMalloc(&s->d_clear, sizeof(int) * S), "server clears");
    CUDA_TRY(cudaMalloc(&s->d_ctr, sizeof(Counters)), "server counters");
    CUDA_TRY(cudaMalloc(&s->d_nf, sizeof(unsigned) * 4 * S), "server direction counts");
    CUDA_TRY(cudaMalloc(&s->d_mf, sizeof(unsigned long long) * 4 * S), "server direction degree sums");
    CUDA_TRY(cudaMalloc(&s->d_dir, sizeof(MsDir) * 2 * S), "server direction states");
    CUDA_TRY(cudaMalloc(&s->d_bu, S), "server bottom-up flags");
    CUDA_TRY(cudaMalloc(&s->d_bu_prefix, sizeof(unsigned) * (S + 1)), "server bottom-up steps");
    CUDA_TRY(cudaHostAlloc(&s->h_ctr, sizeof(Counters), cudaHostAllocDefault), "server pinned counters");
    CUDA_TRY(cudaHostAlloc(&s->h_slots, sizeof(MsSlot) * S, cudaHostAllocDefault), "server pinned slots");
    CUDA_TRY(cudaHostAlloc(&s->h_state, sizeof(MsSlotState) * S, cudaHostAllocDefault), "server pinned states");
    CUDA_TRY(cudaHostAlloc(&s->h_admit, sizeof(int2) * S, cudaHostAllocDefault), "server pinned admissions");
    CUDA_TRY(cudaHostAlloc(&s->h_clear, sizeof(int) * S, cudaHostAllocDefault), "server pinned clears");
    std::memset(s->h_slots, 0, sizeof(MsSlot) * S);
    s->use.assign(S, SlotUse());
    s->free_slots.clear();
    for (int i = int(S) - 1; i >= 0; i--) s->free_slots.push_back(i);
    return B40C_SUCCESS;
}

void fill_params(b40c_server *s) {
    MsParams &p = s->params;
    p = MsParams{};
    p.graphs = s->d_graphs;
    p.slots = s->d_slots;
    p.state = s->d_state;
    p.alive = s->d_alive;
    p.nslots = s->max_slots;
    p.labels = s->d_labels;
    p.mask = s->d_mask;
    p.queue[0] = s->d_queue[0];
    p.queue[1] = s->d_queue[1];
    p.qcap = (long long)s->labels.capacity() + 1;
    for (int i = 0; i < 2; i++) {
        p.chunks[i] = s->d_chunks[i];
        p.wchunks[i] = s->d_wchunks[i];
    }
    p.chunk_cap = int(s->chunk_cap);
    p.wchunk_cap = int(s->wchunk_cap);
    p.ctr = s->d_ctr;
    p.wait_ns = s->wait_ns;
    p.warp_th = s->warp_th;
    p.cta_th = std::max(s->cta_th, s->warp_th);
    p.cull_flags = s->cull_flags;
    p.max_levels = s->epoch_levels;
    p.stop_on_retire = 1;
    p.do_alpha = s->mark_pred ? 0u : s->do_alpha;
    p.do_beta = s->do_beta;
    p.nf = s->d_nf;
    p.mf = s->d_mf;
    p.dir = s->d_dir;
    p.bu = s->d_bu;
    p.bu_prefix = s->d_bu_prefix;
}

// Chunk entries a search of graph g can need in one level (as the batch sizes them).
void chunk_need(const b40c_server *s, const ResidentGraph &g, size_t *c, size_t *w) {
    const long long ct = std::max(1, std::max(s->cta_th, s->warp_th)), wt = std::max(1, s->warp_th);
    *c = size_t(g.edges / chunk_edges<128>() + 2 * (g.edges / ct) + 2);
    *w = size_t(g.edges / WARP_CHUNK + 2 * (g.edges / wt) + 2);
}

int translate(unsigned err) {
    if (err & ERR_BAD_VERTEX) return set_error(B40C_ERR_INVALID_VALUE, "server: vertex id out of range");
    if (err & ERR_BARRIER_TIMEOUT) return set_error(B40C_ERR_LAUNCH_TIMEOUT, "server: grid barrier wait timed out");
    if (err & ERR_OVERFLOW) return set_error(B40C_ERR_INVALID_CONFIGURATION, "server: frontier pool overflow");
    return set_error(B40C_ERR_LAUNCH_TIMEOUT, "server: level loop limit");
}

}  // namespace

extern "C" int b40c_server_create(int mark_predecessors, int max_slots, long long hbm_budget_bytes,
                                  b40c_server_t **out) {
    clear_error();
    if (!out || max_slots < 1 || max_slots > (1 << 20) || hbm_budget_bytes <= 0)
        return set_error(B40C_ERR_INVALID_VALUE, "server_create: invalid arguments");
    b40c_server *s = new (std::nothrow) b40c_server();
    if (!s) return set_error(B40C_ERR_MEMORY_ALLOCATION, "server allocation");
    s->mark_pred = mark_predecessors != 0;
    s->max_slots = max_slots;
    cudaError_t e = cudaGetDevice(&s->device);
    if (!e) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e) {
        delete s;
        return cuda_fail(e, "server creation");
    }
    int rc = server_alloc(s, hbm_budget_bytes);
    if (rc) {
        b40c_server_destroy(s);
        return rc;
    }
    *out = s;
    return B40C_SUCCESS;
}

extern "C" int b40c_server_destroy(b40c_server_t *s) {
    clear_error();
    if (!s) return B40C_SUCCESS;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto &g : s->graphs) {
        cudaFree(g.d_row);
        cudaFree(g.d_col);
        cudaFree(g.d_heavy);
    }
    cudaFree(s->d_graphs);
    cudaFree(s->d_slots);
    cudaFree(s->d_state);
    cudaFree(s->d_alive);
    cudaFree(s->d_labels);
    cudaFree(s->d_mask);
    for (int i = 0; i < 2; i++) {
        cudaFree(s->d_queue[i]);
        cudaFree(s->d_chunks[i]);
        cudaFree(s->d_wchunks[i]);
    }
    cudaFree(s->d_admit);
    cudaFree(s->d_clear);
    cudaFree(s->d_nf);
    cudaFree(s->d_mf);
    cudaFree(s->d_dir);
    cudaFree(s->d_bu);
    cudaFree(s->d_bu_prefix);
    cudaFree(s->d_ctr);
    cudaFreeHost(s->h_ctr);
    cudaFreeHost(s->h_slots);
    cudaFreeHost(s->h_state);
    cudaFreeHost(s->h_admit);
    cudaFreeHost(s->h_clear);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return B40C_SUCCESS;
}

extern "C" int b40c_server_add_graph(b40c_server_t *s, int nodes, int edges, const int *h_col, const int *h_row,
                                     int *graph_id) {
    clear_error();
    if (!s || !graph_id || nodes <= 0 || edges < 0 || !h_row || (edges && !h_col))
        return set_error(B40C_ERR_INVALID_VALUE, "server_add_graph: invalid arguments");
    if (h_row[0] != 0 || h_row[nodes] != edges)
        return set_error(B40C_ERR_INVALID_VALUE, "server_add_graph: row offsets do not span [0, edges]");
    for (int v = 0; v < nodes; v++)
        if (h_row[v + 1] < h_row[v]) return set_error(B40C_ERR_INVALID_VALUE, "server_add_graph: bad row offsets");
    for (int k = 0; k < edges; k++)
        if ((unsigned)h_col[k] >= (unsigned)nodes)
            return set_error(B40C_ERR_INVALID_VALUE, "server_add_graph: column index out of range");
    CUDA_TRY(cudaSetDevice(s->device), "cudaSetDevice");
    ResidentGraph g;
    g.nodes = nodes;
    g.edges = edges;
    // Frees the graph's device arrays if a step below fails before the
    // server owns them.
    struct Unwind {
        ResidentGraph *g;
        bool owned = false;
        ~Unwind() {
            if (owned) return;
            cudaFree(g->d_row);
            cudaFree(g->d_col);
            cudaFree(g->d_heavy);
        }
    } unwind{&g};
    CUDA_TRY(cudaMalloc(&g.d_row, sizeof(int) * (size_t(nodes) + 1)), "server graph row offsets");
    CUDA_TRY(cudaMalloc(&g.d_col, sizeof(int) * (size_t(edges) + 4)), "server graph column indices");
    CUDA_TRY(cudaMemcpy(g.d_row, h_row, sizeof(int) * (size_t(nodes) + 1), cudaMemcpyHostToDevice), "upload");
    CUDA_TRY(cudaMemset(g.d_col + edges, 0, 4 * sizeof(int)), "column padding");
    if (edges) CUDA_TRY(cudaMemcpy(g.d_col, h_col, sizeof(int) * size_t(edges), cudaMemcpyHostToDevice), "upload");
    CUDA_TRY(ms_graph_symmetric(g.d_row, g.d_col, nodes, edges, &g.symmetric), "graph symmetry check");
    if (g.symmetric)
        CUDA_TRY(ms_graph_heavy(g.d_row, g.d_col, nodes, edges, &g.d_heavy), "heaviest-neighbour keys");
    // The new device table (old graphs plus this one) is built and uploaded
    // before it replaces the old one; the server owns the graph only once
    // that succeeded, so a failure leaves s->graphs and s->d_graphs as they were.
    std::vector<MsGraph> table(s->graphs.size() + 1);
    for (size_t i = 0; i < s->graphs.size(); i++)
        table[i] = MsGraph{s->graphs[i].d_row, s->graphs[i].d_col, s->graphs[i].nodes, int(s->graphs[i].edges + 4),
                           int(s->graphs[i].edges), s->graphs[i].symmetric, s->graphs[i].d_heavy};
    table.back() = MsGraph{g.d_row, g.d_col, g.nodes, int(g.edges + 4), int(g.edges), g.symmetric, g.d_heavy};
    MsGraph *d_table = nullptr;
    CUDA_TRY(cudaMalloc(&d_table, sizeof(MsGraph) * table.size()), "server graph table");
    cudaError_t ue = cudaMemcpy(d_table, table.data(), sizeof(MsGraph) * table.size(), cudaMemcpyHostToDevice);
    if (ue != cudaSuccess) {
        cudaFree(d_table);
        CUDA_TRY(ue, "graph table upload");
    }
    cudaFree(s->d_graphs);
    s->d_graphs = d_table;
    s->graphs.push_back(g);
    unwind.owned = true;
    *graph_id = int(s->graphs.size()) - 1;
    return B40C_SUCCESS;
}

extern "C" int b40c_server_set_direction_optimizing(b40c_server_t *s, int alpha, int beta) {
    clear_error();
    if (!s || alpha < 0 || beta < 0 || (alpha > 0 && beta == 0))
        return set_error(B40C_ERR_INVALID_VALUE, "direction switch: alpha >= 0, and beta >= 1 when alpha > 0");
    s->do_alpha = unsigned(alpha);
    s->do_beta = unsigned(beta);
    return B40C_SUCCESS;
}

extern "C" int b40c_server_set_policy(b40c_server_t *s, int cta_threads, int warp_th, int cta_th, int cull_flags,
                                      int epoch_levels) {
    clear_error();
    if (!s) return set_error(B40C_ERR_INVALID_VALUE, "NULL server");
    if (cta_threads && cta_threads != 128 && cta_threads != 256 && cta_threads != 512)
        return set_error(B40C_ERR_INVALID_VALUE, "cta_threads must be 128, 256 or 512");
    if (warp_th < 0 || cta_th < 0 || cull_flags < -1 || cull_flags > 3 || epoch_levels < 0)
        return set_error(B40C_ERR_INVALID_VALUE, "invalid policy field");
    if (cta_threads) s->threads = cta_threads;
    if (warp_th) s->warp_th = warp_th;
    if (cta_th) s->cta_th = cta_th;
    if (cull_flags >= 0) s->cull_flags = unsigned(cull_flags);
    if (epoch_levels) s->epoch_levels = epoch_levels;
    return B40C_SUCCESS;
}

extern "C" int b40c_server_run_trace(b40c_server_t *s, int n, const int *graph_ids, const int *sources,
                                     const double *arrival_us, double *latency_us, int **labels_out,
                                     double *makespan_us) {
    clear_error();
    if (!s || n < 0 || (n && (!graph_ids || !sources || !arrival_us || !latency_us)))
        return set_error(B40C_ERR_INVALID_VALUE, "server_run_trace: invalid arguments");
    for (int i = 0; i < n; i++) {
        if (graph_ids[i] < 0 || graph_ids[i] >= (int)s->graphs.size())
            return set_error(B40C_ERR_INVALID_VALUE, "server_run_trace: query %d names unknown graph %d", i,
                             graph_ids[i]);
        const ResidentGraph &g = s->graphs[graph_ids[i]];
        if (sources[i] < 0 || sources[i] >= g.nodes)
            return set_error(B40C_ERR_INVALID_VALUE, "server_run_trace: query %d source out of range", i);
        if (i && arrival_us[i] < arrival_us[i - 1])
            return set_error(B40C_ERR_INVALID_VALUE, "server_run_trace: arrival times must not decrease");
        size_t c, w;
        chunk_need(s, g, &c, &w);
        if (size_t(g.nodes) > s->labels.capacity() || c > s->chunk_cap || w > s->wchunk_cap)
            return set_error(B40C_ERR_MEMORY_ALLOCATION, "server_run_trace: query %d's graph exceeds the HBM budget",
                             i);
    }
    CUDA_TRY(cudaSetDevice(s->device), "cudaSetDevice");
    MsKernelConfig kc{s->threads, s->mark_pred};
    CUDA_TRY(ms_grid_limit(kc, &s->grid), "multi-search occupancy");
    fill_params(s);
    cudaStream_t st = s->stream;
    // Fresh device state for the trace.
    CUDA_TRY(cudaMemsetAsync(s->d_ctr, 0, sizeof(Counters), st), "counters clear");
    CUDA_TRY(cudaMemsetAsync(s->d_state, 0, sizeof(MsSlotState) * s->max_slots, st), "states clear");
    CUDA_TRY(cudaMemsetAsync(s->d_alive, 0, 4 * size_t(s->max_slots), st), "alive clear");
    CUDA_TRY(cudaStreamSynchronize(st), "server setup");
    s->epochs = 0;
    s->max_active = 0;

    using clock = std::chrono::steady_clock;
    const auto t0 = clock::now();
    auto now_us = [&]() { return std::chrono::duration<double, std::micro>(clock::now() - t0).count(); };
    int next = 0, done = 0, level = 0;  // level: the device's Counters::cur_it between epochs
    std::vector<int> active;
    while (done < n) {
        // Admit every arrived query that fits.
        int nadmit = 0;
        double t = now_us();
        while (next < n && arrival_us[next] <= t && !s->free_slots.empty()) {
            const ResidentGraph &g = s->graphs[graph_ids[next]];
            size_t c, w, loff, moff;
            chunk_need(s, g, &c, &w);
            if (s->chunk_used + c > s->chunk_cap || s->wchunk_used + w > s->wchunk_cap) break;
            if (!s->labels.alloc(size_t(g.nodes), &loff)) break;
            if (!s->masks.alloc(size_t((g.nodes + 31) / 32), &moff)) {
                s->labels.release(loff, size_t(g.nodes));
                break;
            }
            const int slot = s->free_slots.back();
            s->free_slots.pop_back();
            SlotUse &u = s->use[slot];
            u.query = next;
            u.label_off = loff;
            u.mask_off = moff;
            u.chunks = c;
            u.wchunks = w;
            u.nodes = g.nodes;
            s->chunk_used += c;
            s->wchunk_used += w;
            MsSlot d{};
            d.label_off = (long long)loff;
            d.mask_off = (long long)moff;
            d.graph = graph_ids[next];
            d.start_level = 0;  // set on the device side below (current level)
            d.nodes = g.nodes;
            s->h_slots[slot] = d;
            s->h_admit[nadmit] = make_int2(slot, sources[next]);
            s->h_clear[nadmit] = slot;
            nadmit++;
            active.push_back(slot);
            next++;
        }
        if (nadmit) {
            // The current level is the admitted searches' start level.
            for (int k = 0; k < nadmit; k++) s->h_slots[s->h_admit[k].x].start_level = level;
            CUDA_TRY(cudaMemcpyAsync(s->d_slots, s->h_slots, sizeof(MsSlot) * s->max_slots, cudaMemcpyHostToDevice,
                                     st),
                     "slot table upload");
            CUDA_TRY(cudaMemcpyAsync(s->d_clear, s->h_clear, sizeof(int) * nadmit, cudaMemcpyHostToDevice, st),
                     "clear list upload");
            CUDA_TRY(cudaMemcpyAsync(s->d_admit, s->h_admit, sizeof(int2) * nadmit, cudaMemcpyHostToDevice, st),
                     "admission upload");
            CUDA_TRY(ms_clear_slots(s->params, s->d_clear, nadmit, st), "slot clear kernel");
            CUDA_TRY(ms_admit(s->params, kc, s->d_admit, nadmit, st), "admission kernel");
        }
        if (active.empty()) {
            if (next < n) {
                const double wait = arrival_us[next] - now_us();
                if (wait > 200.0) std::this_thread::sleep_for(std::chrono::microseconds(long(wait - 100.0)));
            }
            continue;
        }
        s->max_active = std::max<long long>(s->max_active, (long long)active.size());
        // One epoch of the persistent kernel.
        CUDA_TRY(cudaMemsetAsync(&s->d_ctr->retired, 0, sizeof(s->d_ctr->retired), st), "retired ring clear");
        CUDA_TRY(ms_launch(s->params, kc, s->grid, st), "multi-search kernel launch");
        CUDA_TRY(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(MsSlotState) * s->max_slots, cudaMemcpyDeviceToHost,
                                 st),
                 "state copy");
        CUDA_TRY(cudaMemcpyAsync(s->h_ctr, s->d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st), "counters copy");
        CUDA_TRY(cudaStreamSynchronize(st), "serving epoch");
        s->epochs++;
        if (s->h_ctr->error | s->h_ctr->sticky) return translate(s->h_ctr->error | s->h_ctr->sticky);
        level = s->h_ctr->cur_it;
        // Retire finished searches.
        const double tc = now_us();
        for (size_t k = 0; k < active.size();) {
            const int slot = active[k];
            if (s->h_state[slot].active) {
                k++;
                continue;
            }
            SlotUse &u = s->use[slot];
            const long long q = u.query;
            latency_us[q] = tc - arrival_us[q];
            if (labels_out && labels_out[q])
                CUDA_TRY(cudaMemcpy(labels_out[q], s->d_labels + u.label_off, sizeof(int) * size_t(u.nodes),
                                    cudaMemcpyDeviceToHost),
                         "result copy");
            s->labels.release(u.label_off, size_t(u.nodes));
            s->masks.release(u.mask_off, size_t((u.nodes + 31) / 32));
            s->chunk_used -= u.chunks;
            s->wchunk_used -= u.wchunks;
            u = SlotUse();
            s->free_slots.push_back(slot);
            active[k] = active.back();
            active.pop_back();
            done++;
        }
    }
    if (makespan_us) *makespan_us = now_us();
    return B40C_SUCCESS;
}

extern "C" int b40c_server_stats(b40c_server_t *s, long long *epochs, long long *max_active) {
    clear_error();
    if (!s) return set_error(B40C_ERR_INVALID_VALUE, "NULL server");
    if (epochs) *epochs = s->epochs;
    if (max_active) *max_active = s->max_active;
    return B40C_SUCCESS;
}
