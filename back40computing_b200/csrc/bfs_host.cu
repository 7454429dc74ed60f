// Host orchestration and C ABI of libb40c_bfs: CsrProblem and the enactors.
//
// b40c_problem mirrors bfs::CsrProblem<int,int,MARK_PREDECESSORS>
// (b40c/graph/bfs/csr_problem.cuh:68-751) for one GPU: it owns the device CSR,
// labels, visited mask and frontier queues.  b40c_enactor mirrors the
// Enactor{ExpandContract,ContractExpand,TwoPhase} classes: it owns the search
// counters, the two grid-wide chunk tables, its stream, timing events, the cached
// per-level CUDA graph.  Each entry point returns a cudaError_t value and
// records a message in the thread's error slot (B40CPerror,
// b40c/util/error_utils.cuh:44-103).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "b40c_bfs.h"
#include "bfs_kernels.cuh"
#include "host_common.h"

namespace b40c_b200 {

static thread_local char g_error[512];

int set_error(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    if (code && getenv("B40C_VERBOSE_ERRORS")) fprintf(stderr, "[b40c_bfs] %s (error %d)\n", g_error, code);
    return code;
}
void clear_error() { g_error[0] = 0; }
const char *last_error() { return g_error; }

static int cuda_fail(cudaError_t e, const char *what) {
    return set_error(int(e), "%s failed (CUDA error %d: %s)", what, int(e), cudaGetErrorString(e));
}
#define CUDA_TRY(call, what)                            \
    do {                                                \
        cudaError_t _e = (call);                        \
        if (_e != cudaSuccess) return cuda_fail(_e, what); \
    } while (0)

}  // namespace b40c_b200

using namespace b40c_b200;

struct b40c_problem {
    int device = 0;
    bool mark_pred = false;
    int64_t nodes = 0, edges = 0;
    bool mapped = false;  // stream_from_host
    std::vector<void *> registered;
    int *d_row_offsets = nullptr;
    int *d_col = nullptr;
    int *d_labels = nullptr;
    unsigned *d_mask = nullptr;
    size_t mask_bytes = 0;
    size_t col_cap = 0, row_cap = 0, labels_cap = 0, mask_cap = 0;  // device allocations kept across uploads
    int *d_queue[2] = {nullptr, nullptr};
    int *d_pred[2] = {nullptr, nullptr};
    long long queue_elems[2] = {0, 0};
    long long pred_elems[2] = {0, 0};
    bool reset_once = false;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int symmetric = -1;                    // -1 unknown, 0 no, 1 yes (checked on first use)
    unsigned long long *d_sym = nullptr;   // 4 hash sums of the symmetry check
    unsigned *d_mask_snap = nullptr;       // predecessor-label bottom-up levels: visited-mask copy
    size_t mask_snap_cap = 0;
    unsigned long long *d_heavy = nullptr;  // bottom-up levels: per vertex, its neighbour of highest degree
    size_t heavy_cap = 0;
    bool heavy_ready = false;               // d_heavy holds the current graph's keys
    // Two label buffers (b40c_problem_set_label_buffers): each Reset switches
    // to the other one, and ExtractResultsAsync copies on a side stream, so
    // the copy of one search's labels to the host overlaps the next search.
    int label_buffers = 1;
    int *d_labels_alt = nullptr;
    size_t labels_alt_cap = 0;
    bool use_alt = false;                        // the current labels are in d_labels_alt
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t after_search = nullptr;          // problem-stream point a side copy waits for
    cudaEvent_t copied[2] = {nullptr, nullptr};  // the last side copy out of d_labels / d_labels_alt
};

struct b40c_enactor {
    int device = 0;
    int strategy = B40C_EXPAND_CONTRACT;
    bool instrument = false, debug = false;
    int threads = 256;
    int warp_th = 64, cta_th = 1024;
    unsigned cull_flags = CULL_HISTORY;
    unsigned do_alpha = 0, do_beta = 0;  // direction-optimizing expand-contract (0: top-down only)
    unsigned long long wait_ns = 5000000000ull;
    int l2_persist = 0;  // b40c_enactor_set_l2_persistence
    bool stage_bu = false;  // b40c_enactor_set_bottom_up_staging
    int narrow_team = 0;       // b40c_enactor_set_narrow_levels: cluster CTAs asked for (0: off)
    unsigned narrow_max = 0;   // and its frontier bound
    unsigned flat_max = 0;     // full-grid levels with the latency-first body (0: none)
    int narrow_key = -1;       // launch configuration narrow_got was found for
    int narrow_got = 0;        // the cluster size used (0: none fits)
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    Counters *d_ctr = nullptr;
    Counters *h_ctr = nullptr;  // pinned
    int4 *d_chunks[2] = {nullptr, nullptr};   // CTA chunks
    int4 *d_wchunks[2] = {nullptr, nullptr};  // warp chunks
    int chunk_cap = 0;   // entries per CTA chunk table
    int wchunk_cap = 0;  // entries per warp chunk table
    LevelRecord *d_levels = nullptr;  // per-level log, when enabled
    bool log_levels = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    int last_iteration = 0;
    long long last_total_queued = 0;
    double last_duty = 0.0;
    unsigned long long *d_busy = nullptr;  // INSTRUMENT: per-CTA busy ns of the last fused search
    int busy_cap = 0;
    int busy_grid = 0;  // CTAs of the last instrumented fused search (0: none)
    bool have_stats = false;
    bool timing_pending = false;
    // Cached per-level graphs, two of them (a problem with two label buffers
    // alternates its labels pointer between searches); the most recently used
    // one is entry 0.
    struct LevelGraph {
        cudaGraphExec_t exec = nullptr;
        cudaGraph_t graph = nullptr;
        BfsParams params{};
        KernelConfig kc{};
        int grid = 0;
    } lg[2];
};

namespace {

constexpr int LEVEL_LOG_CAP = 4096;

cudaStream_t problem_stream(b40c_problem *p) { return p->stream ? p->stream : p->own_stream; }
// The label buffer the last Reset initialised: searches write it, extracts read it.
int *cur_labels(const b40c_problem *p) { return p->use_alt ? p->d_labels_alt : p->d_labels; }
// Waits for everything queued on the problem: its stream and side-stream label copies.
void sync_problem(b40c_problem *p) {
    cudaStreamSynchronize(problem_stream(p));
    if (p->copy_stream) cudaStreamSynchronize(p->copy_stream);
}
cudaStream_t enactor_stream(b40c_enactor *e) { return e->stream ? e->stream : e->own_stream; }

// The ends of the row offsets, checked on the host; the rest of the CSR
// (offsets that decrease, column ids out of range) is checked on the device
// after the upload (device_check_csr).
int check_csr_ends(int64_t nodes, int64_t edges, const int *row) {
    if (row[0] != 0) return set_error(B40C_ERR_INVALID_VALUE, "CSR row_offsets[0] = %d, expected 0", row[0]);
    if (row[nodes] != edges)
        return set_error(B40C_ERR_INVALID_VALUE, "CSR row_offsets[nodes] = %d, expected edges = %lld",
                         row[nodes], (long long)edges);
    return B40C_SUCCESS;
}

void unmap_host(b40c_problem *p);

void free_problem_device(b40c_problem *p) {
    if (!p->mapped) {
        cudaFree(p->d_row_offsets);
        cudaFree(p->d_col);
    }
    unmap_host(p);
    p->d_row_offsets = nullptr;
    p->d_col = nullptr;
    p->col_cap = p->row_cap = 0;
    cudaFree(p->d_labels);
    cudaFree(p->d_labels_alt);
    cudaFree(p->d_mask);
    p->d_labels = p->d_labels_alt = nullptr;
    p->d_mask = nullptr;
    p->labels_cap = p->labels_alt_cap = p->mask_cap = 0;
    p->use_alt = false;
    for (int i = 0; i < 2; i++) {
        cudaFree(p->d_queue[i]);
        cudaFree(p->d_pred[i]);
        p->d_queue[i] = p->d_pred[i] = nullptr;
        p->queue_elems[i] = p->pred_elems[i] = 0;
    }
    cudaFree(p->d_sym);
    p->d_sym = nullptr;
    p->symmetric = -1;
    cudaFree(p->d_mask_snap);
    p->d_mask_snap = nullptr;
    p->mask_snap_cap = 0;
    cudaFree(p->d_heavy);
    p->d_heavy = nullptr;
    p->heavy_cap = 0;
    p->heavy_ready = false;
}

// Whether every entry v of row u has an entry u in row v (a symmetric,
// undirected graph), which bottom-up levels need.  Decided once per graph by
// two 64-bit hash sums over the entries and their reverses (a non-symmetric
// graph passes only on a double 64-bit collision), with a host wait.
int ensure_symmetry_known(b40c_problem *p) {
    if (p->symmetric >= 0) return B40C_SUCCESS;
    cudaStream_t s = problem_stream(p);
    if (!p->d_sym) CUDA_TRY(cudaMalloc(&p->d_sym, 4 * sizeof(unsigned long long)), "cudaMalloc symmetry sums");
    unsigned long long h[4] = {0, 0, 0, 0};
    CUDA_TRY(cudaMemsetAsync(p->d_sym, 0, sizeof(h), s), "symmetry sums clear");
    CUDA_TRY(launch_symmetry_hash(p->d_row_offsets, p->d_col, int(p->nodes), p->edges, p->d_sym, s),
             "symmetry check launch");
    CUDA_TRY(cudaMemcpyAsync(h, p->d_sym, sizeof(h), cudaMemcpyDeviceToHost, s), "symmetry sums copy");
    CUDA_TRY(cudaStreamSynchronize(s), "symmetry check");
    p->symmetric = (h[0] == h[1] && h[2] == h[3]) ? 1 : 0;
    return B40C_SUCCESS;
}

// Per vertex, its neighbour of highest degree (launch_heavy_neighbour), which
// bottom-up levels probe before reading a list.  Built once per graph on the
// problem's stream, with a host wait, like the symmetry check.
int ensure_heavy_known(b40c_problem *p) {
    if (p->heavy_ready) return B40C_SUCCESS;
    cudaStream_t s = problem_stream(p);
    // HEAVY_PAD zero keys past the last vertex: a bottom-up step stages whole
    // 16-byte units of keys with one bulk copy.
    const size_t keys = size_t(p->nodes) + HEAVY_PAD;
    if (p->heavy_cap < keys) {
        cudaFree(p->d_heavy);
        p->d_heavy = nullptr;
        p->heavy_cap = 0;
        CUDA_TRY(cudaMalloc(&p->d_heavy, sizeof(unsigned long long) * keys), "cudaMalloc heaviest-neighbour keys");
        p->heavy_cap = keys;
    }
    CUDA_TRY(cudaMemsetAsync(p->d_heavy, 0, sizeof(unsigned long long) * keys, s), "heaviest-neighbour keys clear");
    CUDA_TRY(launch_heavy_neighbour(p->d_row_offsets, p->d_col, int(p->nodes), p->edges, p->d_heavy, s),
             "heaviest-neighbour launch");
    CUDA_TRY(cudaStreamSynchronize(s), "heaviest-neighbour keys");
    p->heavy_ready = true;
    return B40C_SUCCESS;
}

// Checks the uploaded CSR on the device (rows whose offsets decrease, column
// ids outside [0, nodes)) and reports the first fault as the host check
// would, reading the offending values from the caller's arrays.
int device_check_csr(b40c_problem *p, const int *h_row, const int *h_col) {
    cudaStream_t s = problem_stream(p);
    if (!p->d_sym) CUDA_TRY(cudaMalloc(&p->d_sym, 4 * sizeof(unsigned long long)), "cudaMalloc check buffer");
    unsigned long long h[2];
    CUDA_TRY(cudaMemsetAsync(p->d_sym, 0xff, sizeof(h), s), "CSR check clear");
    CUDA_TRY(launch_csr_check(p->d_row_offsets, p->d_col, int(p->nodes), p->edges, p->d_sym, s), "CSR check launch");
    CUDA_TRY(cudaMemcpyAsync(h, p->d_sym, sizeof(h), cudaMemcpyDeviceToHost, s), "CSR check copy");
    CUDA_TRY(cudaStreamSynchronize(s), "CSR check");
    if (h[0] != ~0ull)
        return set_error(B40C_ERR_INVALID_VALUE, "CSR row_offsets decrease at row %lld", (long long)h[0]);
    if (h[1] != ~0ull)
        return set_error(B40C_ERR_INVALID_VALUE, "CSR column index %d at edge %lld outside [0, %lld)",
                         h_col[h[1]], (long long)h[1], (long long)p->nodes);
    return B40C_SUCCESS;
}

// Host ranges this library registered for stream_from_host, with the number
// of problems using each.  Several problems may map the same caller arrays;
// the range is unregistered when the last of them lets go.  Memory the
// caller pinned itself (cudaHostAlloc, or registered outside the library) is
// never registered or unregistered here.
std::mutex g_reg_mutex;
std::map<void *, int> g_registrations;

int map_host(b40c_problem *p, const void *h, size_t bytes, void **d) {
    void *ptr = const_cast<void *>(h);
    {
        std::lock_guard<std::mutex> lock(g_reg_mutex);
        auto it = g_registrations.find(ptr);
        if (it != g_registrations.end()) {
            it->second++;
            p->registered.push_back(ptr);
        } else {
            cudaPointerAttributes attr{};
            cudaError_t e = cudaPointerGetAttributes(&attr, h);
            if (e != cudaSuccess) cudaGetLastError();
            if (e != cudaSuccess || attr.type != cudaMemoryTypeHost) {
                e = cudaHostRegister(ptr, bytes, cudaHostRegisterMapped | cudaHostRegisterReadOnly);
                if (e != cudaSuccess) return cuda_fail(e, "CsrProblem cudaHostRegister (stream_from_host)");
                g_registrations[ptr] = 1;
                p->registered.push_back(ptr);
            }
        }
    }
    CUDA_TRY(cudaHostGetDevicePointer(d, ptr, 0), "CsrProblem cudaHostGetDevicePointer");
    return B40C_SUCCESS;
}

void unmap_host(b40c_problem *p) {
    std::lock_guard<std::mutex> lock(g_reg_mutex);
    for (void *h : p->registered) {
        auto it = g_registrations.find(h);
        if (it != g_registrations.end() && --it->second == 0) {
            cudaHostUnregister(h);
            g_registrations.erase(it);
        }
    }
    p->registered.clear();
}

int translate_device_error(unsigned err) {
    if (err & ERR_BAD_VERTEX)
        return set_error(B40C_ERR_INVALID_VALUE, "column index outside [0, nodes) met during the search");
    if (err & ERR_BARRIER_TIMEOUT)
        return set_error(B40C_ERR_LAUNCH_TIMEOUT,
                         "grid barrier wait exceeded its limit; search abandoned (context still usable)");
    if (err & ERR_LEVEL_LIMIT)
        return set_error(B40C_ERR_LAUNCH_TIMEOUT, "level loop passed nodes + 2 levels; search abandoned");
    if (err & ERR_OVERFLOW)
        return set_error(B40C_ERR_INVALID_CONFIGURATION,
                         "Frontier queue overflow.  Please increase queue-sizing factor.");
    return B40C_SUCCESS;
}

int ensure_enactor_buffers(b40c_enactor *e, b40c_problem *p) {
    if (!e->d_ctr) {
        CUDA_TRY(cudaMalloc(&e->d_ctr, sizeof(Counters)), "Enactor cudaMalloc counters");
        CUDA_TRY(cudaMemset(e->d_ctr, 0, sizeof(Counters)), "Enactor cudaMemset counters");
        CUDA_TRY(cudaHostAlloc(&e->h_ctr, sizeof(Counters), cudaHostAllocDefault), "Enactor cudaHostAlloc");
        std::memset(e->h_ctr, 0, sizeof(Counters));
    }
    // Chunks per phase: each vertex expands once per search, and a list of len
    // edges placed in a table of CH-edge chunks takes at most len / CH + 2
    // entries (CH >= 2048 for CTA chunks, 512 for warp chunks).
    const long long ct = std::max(1, std::max(e->cta_th, e->warp_th)), wt = std::max(1, e->warp_th);
    long long need = p->edges / chunk_edges<128>() + 2 * (p->edges / ct) + 64;
    long long wneed = p->edges / WARP_CHUNK + 2 * (p->edges / wt) + 64;
    need = std::min(need, 1ll << 30);
    wneed = std::min(wneed, 1ll << 30);
    if (e->chunk_cap < need) {
        for (int i = 0; i < 2; i++) {
            cudaFree(e->d_chunks[i]);
            e->d_chunks[i] = nullptr;
        }
        e->chunk_cap = 0;
        for (int i = 0; i < 2; i++)
            CUDA_TRY(cudaMalloc(&e->d_chunks[i], sizeof(int4) * size_t(need)), "Enactor cudaMalloc CTA chunk table");
        e->chunk_cap = int(need);
    }
    if (e->wchunk_cap < wneed) {
        for (int i = 0; i < 2; i++) {
            cudaFree(e->d_wchunks[i]);
            e->d_wchunks[i] = nullptr;
        }
        e->wchunk_cap = 0;
        for (int i = 0; i < 2; i++)
            CUDA_TRY(cudaMalloc(&e->d_wchunks[i], sizeof(int4) * size_t(wneed)), "Enactor cudaMalloc warp chunk table");
        e->wchunk_cap = int(wneed);
    }
    if (e->log_levels && !e->d_levels)
        CUDA_TRY(cudaMalloc(&e->d_levels, sizeof(LevelRecord) * LEVEL_LOG_CAP), "Enactor cudaMalloc level log");
    return B40C_SUCCESS;
}

// Whether a column array of `edges` entries is streamed with evict_first:
// when it takes more than a quarter of the device's L2.
bool stream_column(int device, int64_t edges) {
    int l2 = 0;
    if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device) != cudaSuccess || l2 <= 0) return true;
    return double(edges) * sizeof(int) > 0.25 * double(l2);
}

int fill_params(b40c_enactor *e, b40c_problem *p, int src, BfsParams &bp) {
    bp = BfsParams{};
    bp.row_offsets = p->d_row_offsets;
    bp.col = p->d_col;
    bp.labels = cur_labels(p);
    bp.mask = p->d_mask;
    for (int i = 0; i < 2; i++) {
        bp.queue[i] = p->d_queue[i];
        bp.pred_queue[i] = p->d_pred[i];
    }
    bp.chunks[0] = e->d_chunks[0];
    bp.chunks[1] = e->d_chunks[1];
    bp.wchunks[0] = e->d_wchunks[0];
    bp.wchunks[1] = e->d_wchunks[1];
    bp.levels = e->log_levels ? e->d_levels : nullptr;
    bp.level_cap = LEVEL_LOG_CAP;
    bp.ctr = e->d_ctr;
    bp.wait_ns = e->wait_ns;
    long long qcap = std::min(p->queue_elems[0], p->queue_elems[1]);
    if (p->mark_pred && e->strategy != B40C_EXPAND_CONTRACT)
        qcap = std::min(qcap, std::min(p->pred_elems[0], p->pred_elems[1]));
    if (qcap > 0xffffffffll) qcap = 0xffffffffll;
    bp.qcap = qcap;
    bp.chunk_cap = e->chunk_cap;
    bp.wchunk_cap = e->wchunk_cap;
    bp.vec_end = p->mapped ? int(p->edges & ~int64_t(3)) : int(p->edges + 4);
    bp.nodes = int(p->nodes);
    bp.src = src;
    bp.warp_th = e->warp_th;
    bp.cta_th = std::max(e->cta_th, e->warp_th);
    bp.cull_flags = e->cull_flags;
    bp.edges = p->edges;
    bp.stream_col = stream_column(p->device, p->edges) ? 1 : 0;
    bp.count_raw = e->instrument ? 1 : 0;
    bp.do_alpha = 0;  // enabled by enqueue_search for searches that can run bottom-up
    bp.do_beta = 0;
    if (qcap < 1) return set_error(B40C_ERR_ILLEGAL_STATE, "frontier queues not allocated: call Reset first");
    if (p->mark_pred && e->strategy != B40C_EXPAND_CONTRACT && (!p->d_pred[0] || !p->d_pred[1]))
        return set_error(B40C_ERR_ILLEGAL_STATE,
                         "predecessor queues missing: Reset with this enactor's frontier type");
    return B40C_SUCCESS;
}

int set_persist_window(b40c_enactor *e, b40c_problem *p, cudaStream_t s, bool on);
int launch_search(b40c_enactor *e, BfsParams &bp, const KernelConfig &kc, cudaStream_t s, int max_grid_size,
                  int variant);

int enqueue_search(b40c_enactor *e, b40c_problem *p, int src, int max_grid_size, int variant) {
    if (!e || !p) return set_error(B40C_ERR_INVALID_VALUE, "NULL enactor or problem");
    if (!p->d_col || !cur_labels(p) || !p->reset_once)
        return set_error(B40C_ERR_ILLEGAL_STATE, "problem needs FromHostProblem and Reset before a search");
    if (src < 0 || src >= p->nodes)
        return set_error(B40C_ERR_INVALID_VALUE, "source %d outside [0, %lld)", src, (long long)p->nodes);
    int rc = ensure_enactor_buffers(e, p);
    if (rc) return rc;
    BfsParams bp;
    if ((rc = fill_params(e, p, src, bp))) return rc;
    KernelConfig kc{e->strategy, e->threads, p->mark_pred};
    cudaStream_t s = enactor_stream(e);
    // The problem's pending work (Reset) precedes the search.
    cudaStream_t ps = problem_stream(p);
    if (ps != s) {
        cudaEvent_t dep;
        CUDA_TRY(cudaEventCreateWithFlags(&dep, cudaEventDisableTiming), "cudaEventCreate");
        cudaEventRecord(dep, ps);
        cudaStreamWaitEvent(s, dep, 0);
        cudaEventDestroy(dep);
    }
    if (variant < B40C_VARIANT_DEFAULT || variant > B40C_VARIANT_ITERATIVE)
        return set_error(B40C_ERR_INVALID_VALUE, "unknown variant %d", variant);
    // The hybrid switches between its two bodies inside one persistent launch;
    // like the reference's EnactorHybrid it has a single way to run a search.
    if (variant == B40C_VARIANT_DEFAULT || e->strategy == B40C_HYBRID) variant = B40C_VARIANT_FUSED;
    // Bottom-up levels: fused expand-contract on a symmetric graph held on the
    // device (their scattered column reads would cross PCIe one entry at a time
    // from a stream_from_host graph); with predecessor labels they probe a copy
    // of the visited mask.
    if (e->strategy == B40C_EXPAND_CONTRACT && variant == B40C_VARIANT_FUSED && e->do_alpha && !p->mapped) {
        if ((rc = ensure_symmetry_known(p))) return rc;
        if (p->symmetric == 1) {
            if (p->mark_pred && p->mask_snap_cap < p->mask_bytes) {
                cudaFree(p->d_mask_snap);
                p->d_mask_snap = nullptr;
                p->mask_snap_cap = 0;
                CUDA_TRY(cudaMalloc(&p->d_mask_snap, p->mask_bytes), "cudaMalloc visited-mask copy");
                p->mask_snap_cap = p->mask_bytes;
            }
            if ((rc = ensure_heavy_known(p))) return rc;
            bp.mask_snap = p->d_mask_snap;
            bp.heavy = p->d_heavy;
            bp.stage_bu = e->stage_bu ? 1 : 0;  // the problem's row offsets, mask and keys carry the padding
            kc.stage_bu = e->stage_bu;           // and the launch carries the stage buffers
            bp.do_alpha = e->do_alpha;
            bp.do_beta = e->do_beta;
        }
    }
    if (bp.levels)
        CUDA_TRY(cudaMemsetAsync(bp.levels, 0, sizeof(LevelRecord) * LEVEL_LOG_CAP, s), "level log clear");
    if (e->l2_persist && (rc = set_persist_window(e, p, s, true))) return rc;
    rc = launch_search(e, bp, kc, s, max_grid_size, variant);
    if (e->l2_persist) {
        const int rc2 = set_persist_window(e, p, s, false);
        if (!rc) rc = rc2;
    }
    return rc;
}

// The persisting access-policy window of b40c_enactor_set_l2_persistence on
// stream s: the visited mask (what 1), or the mask and the labels when their
// two allocations lie side by side (what 2); on = false clears it.
int set_persist_window(b40c_enactor *e, b40c_problem *p, cudaStream_t s, bool on) {
    cudaStreamAttrValue v{};
    if (on) {
        int max_window = 0, max_persist = 0;
        CUDA_TRY(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, p->device),
                 "access-policy window size query");
        CUDA_TRY(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, p->device),
                 "persisting L2 size query");
        char *lo = reinterpret_cast<char *>(p->d_mask);
        char *hi = lo + p->mask_bytes;
        if (e->l2_persist == 2) {
            char *l = reinterpret_cast<char *>(cur_labels(p));
            char *lh = l + sizeof(int) * size_t(p->nodes);
            char *a = std::min(lo, l), *z = std::max(hi, lh);
            const size_t both = size_t(hi - lo) + size_t(lh - l);
            if (size_t(z - a) <= size_t(max_window) && size_t(z - a) <= both + (size_t(1) << 20)) {
                lo = a;
                hi = z;
            }
        }
        const size_t bytes = std::min(size_t(hi - lo), size_t(max_window));
        size_t limit = 0;
        CUDA_TRY(cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize), "persisting L2 limit query");
        const size_t want = std::min(bytes, size_t(max_persist));
        if (limit < want) CUDA_TRY(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want), "persisting L2 limit");
        v.accessPolicyWindow.base_ptr = lo;
        v.accessPolicyWindow.num_bytes = bytes;
        v.accessPolicyWindow.hitRatio = bytes ? std::min(1.0f, float(double(want) / double(bytes))) : 0.f;
        v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    }
    CUDA_TRY(cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &v), "access-policy window");
    return B40C_SUCCESS;
}

// The launches of one search on stream s (init kernel, then the fused kernel
// or the per-level graph), bracketed by the enactor's timing events.
int launch_search(b40c_enactor *e, BfsParams &bp, const KernelConfig &kc, cudaStream_t s, int max_grid_size,
                  int variant) {
    CUDA_TRY(cudaEventRecord(e->ev0, s), "cudaEventRecord");
    CUDA_TRY(launch_search_init(bp, kc, s), "search init kernel launch");
    if (variant == B40C_VARIANT_FUSED) {
        int limit = 0;
        CUDA_TRY(fused_grid_limit(kc, &limit), "occupancy query");
        int grid = max_grid_size > 0 ? std::min(max_grid_size, limit) : limit;
        e->busy_grid = 0;
        if (e->instrument) {
            if (e->busy_cap < grid) {
                cudaFree(e->d_busy);
                e->d_busy = nullptr;
                e->busy_cap = 0;
                CUDA_TRY(cudaMalloc(&e->d_busy, sizeof(unsigned long long) * size_t(grid)), "cudaMalloc duty stats");
                e->busy_cap = grid;
            }
            bp.cta_busy = e->d_busy;
            e->busy_grid = grid;
        }
        if (kc.strategy == B40C_CONTRACT_EXPAND || kc.strategy == B40C_HYBRID) bp.flat_max = e->flat_max;
        if (e->narrow_team > 0) {
            // the launch's shared memory depends on all but the team: a new
            // configuration is checked (and opted in) before its first launch
            const int key = (kc.threads << 8) | (kc.mark_pred ? 128 : 0) | (kc.stage_bu ? 64 : 0) | e->narrow_team;
            if (e->narrow_key != key) {
                CUDA_TRY(narrow_team_limit(kc, e->narrow_team, &e->narrow_got), "cluster occupancy query");
                e->narrow_key = key;
            }
            if (e->narrow_got > 0) {
                bp.narrow_max = e->narrow_max;
                // The hybrid runs a level above 4 edges per grid thread as two
                // phases: its narrow levels stay below that.
                if (kc.strategy == B40C_HYBRID)
                    bp.narrow_max = unsigned(std::min<long long>(bp.narrow_max, 4ll * kc.threads * grid));
                CUDA_TRY(launch_narrow(bp, kc, e->narrow_got, s), "cluster launch of the narrow BFS kernel");
            }
        }
        CUDA_TRY(launch_fused(bp, kc, grid, s), "cooperative launch of the fused BFS kernel");
    } else if (variant == B40C_VARIANT_ITERATIVE) {
        int limit = 0;
        CUDA_TRY(level_grid_limit(kc, &limit), "occupancy query");
        int grid = max_grid_size > 0 ? std::min(max_grid_size, limit) : limit;
        // A cached graph serves any source: only the init kernel, launched
        // outside the graph, reads it.
        int hit = -1;
        for (int k = 0; k < 2 && hit < 0; k++) {
            const auto &g = e->lg[k];
            BfsParams key = bp;
            key.cond_handle = g.params.cond_handle;
            key.src = g.params.src;
            if (g.exec && g.grid == grid && g.kc.strategy == kc.strategy && g.kc.threads == kc.threads &&
                g.kc.mark_pred == kc.mark_pred && std::memcmp(&key, &g.params, sizeof(BfsParams)) == 0)
                hit = k;
        }
        if (hit < 0) {  // build into entry 1 (the older one), then make it the newest
            auto &g = e->lg[1];
            if (g.exec) cudaGraphExecDestroy(g.exec);
            if (g.graph) cudaGraphDestroy(g.graph);
            g.exec = nullptr;
            g.graph = nullptr;
            BfsParams gp = bp;
            CUDA_TRY(build_level_graph(gp, kc, grid, &g.exec, &g.graph), "building the per-level BFS graph");
            g.params = gp;
            g.kc = kc;
            g.grid = grid;
            hit = 1;
        }
        if (hit == 1) std::swap(e->lg[0], e->lg[1]);
        CUDA_TRY(cudaGraphLaunch(e->lg[0].exec, s), "cudaGraphLaunch");
    } else {
        return set_error(B40C_ERR_INVALID_VALUE, "unknown variant %d", variant);
    }
    CUDA_TRY(cudaEventRecord(e->ev1, s), "cudaEventRecord");
    CUDA_TRY(cudaMemcpyAsync(e->h_ctr, e->d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s),
             "counters copy");
    e->timing_pending = true;
    e->have_stats = false;
    return B40C_SUCCESS;
}

// Waits for the enactor stream; reads counters, timing and the sticky error.
int finish_search(b40c_enactor *e) {
    cudaStream_t s = enactor_stream(e);
    CUDA_TRY(cudaStreamSynchronize(s), "BFS search");
    if (e->timing_pending) {
        cudaEventElapsedTime(&e->last_ms, e->ev0, e->ev1);
        e->timing_pending = false;
    }
    e->last_iteration = e->h_ctr->iteration;
    e->last_total_queued = (long long)e->h_ctr->total_queued;
    e->last_duty = 0.0;
    if (e->busy_grid > 0) {
        // avg_duty as the reference accumulates it (kernel_runtime_stats.cuh:
        // Accumulate): the CTAs' busy times over the longest one times the grid.
        std::vector<unsigned long long> busy(size_t(e->busy_grid));
        CUDA_TRY(cudaMemcpy(busy.data(), e->d_busy, sizeof(unsigned long long) * busy.size(), cudaMemcpyDeviceToHost),
                 "duty stats copy");
        unsigned long long total = 0, longest = 0;
        for (unsigned long long b : busy) {
            total += b;
            longest = std::max(longest, b);
        }
        e->last_duty = longest ? double(total) / (double(longest) * double(busy.size())) : 0.0;
    }
    e->have_stats = true;
    unsigned err = e->h_ctr->sticky | e->h_ctr->error;
    if (err) {
        CUDA_TRY(cudaMemsetAsync(&e->d_ctr->sticky, 0, sizeof(unsigned), s), "clear sticky error");
        CUDA_TRY(cudaStreamSynchronize(s), "clear sticky error");
        e->h_ctr->sticky = 0;
        return translate_device_error(err);
    }
    return B40C_SUCCESS;
}

}  // namespace

// ---- library ----------------------------------------------------------------------------

extern "C" const char *b40c_last_error_string(void) { return last_error(); }
extern "C" const char *b40c_version(void) { return "b40c-bfs-b200 0.1 (sm_100a)"; }

// ---- CsrProblem -----------------------------------------------------------------------

extern "C" int b40c_problem_create(int mark_predecessors, b40c_problem_t **out) {
    clear_error();
    if (!out) return set_error(B40C_ERR_INVALID_VALUE, "NULL out");
    b40c_problem *p = new (std::nothrow) b40c_problem();
    if (!p) return set_error(B40C_ERR_MEMORY_ALLOCATION, "problem allocation");
    p->mark_pred = mark_predecessors != 0;
    cudaError_t e = cudaGetDevice(&p->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete p;
        return cuda_fail(e, "CsrProblem stream creation");
    }
    *out = p;
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_destroy(b40c_problem_t *p) {
    clear_error();
    if (!p) return B40C_SUCCESS;
    cudaSetDevice(p->device);
    sync_problem(p);
    free_problem_device(p);
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
    if (p->after_search) cudaEventDestroy(p->after_search);
    for (cudaEvent_t ev : p->copied)
        if (ev) cudaEventDestroy(ev);
    if (p->own_stream) cudaStreamDestroy(p->own_stream);
    delete p;
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_from_host(b40c_problem_t *p, int stream_from_host, int nodes, int edges,
                                      const int *h_col, const int *h_row, int num_gpus) {
    clear_error();
    if (!p || nodes <= 0 || edges < 0 || !h_row || (edges > 0 && !h_col))
        return set_error(B40C_ERR_INVALID_VALUE, "FromHostProblem: invalid arguments");
    if (num_gpus > 1)
        return set_error(B40C_ERR_NOT_SUPPORTED, "FromHostProblem: multi-GPU slices are not provided");
    if (edges > INT32_MAX - 8192)
        return set_error(B40C_ERR_INVALID_VALUE, "FromHostProblem: %d edges too many for int32 SizeT", edges);
    int rc = check_csr_ends(nodes, edges, h_row);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(p->device), "cudaSetDevice");
    sync_problem(p);
    const bool was_mapped = p->mapped;
    p->mapped = stream_from_host != 0 && edges > 0;
    if (p->mapped || was_mapped) {
        free_problem_device(p);  // mapped arrays are the caller's; device copies are not reused across modes
    } else {
        // A new upload into the same problem reuses its device buffers when they are large enough.
        if (p->labels_cap < size_t(nodes)) {
            cudaFree(p->d_labels);
            p->d_labels = nullptr;
            p->labels_cap = 0;
        }
        if (p->labels_alt_cap < size_t(nodes)) {
            cudaFree(p->d_labels_alt);
            p->d_labels_alt = nullptr;
            p->labels_alt_cap = 0;
        }
        if (p->mask_cap < size_t((nodes + 31) / 32) * 4 + MASK_PAD_BYTES) {
            cudaFree(p->d_mask);
            p->d_mask = nullptr;
            p->mask_cap = 0;
        }
    }
    p->nodes = nodes;
    p->edges = edges;
    p->reset_once = false;
    p->symmetric = -1;
    p->heavy_ready = false;
    if (p->mapped) {
        if ((rc = map_host(p, h_row, sizeof(int) * (size_t(nodes) + 1), (void **)&p->d_row_offsets))) return rc;
        if ((rc = map_host(p, h_col, sizeof(int) * size_t(edges), (void **)&p->d_col))) return rc;
    } else {
        // Column array padded with 4 entries for 16-byte tail loads.
        if (p->col_cap < size_t(edges) + 4) {
            cudaFree(p->d_col);
            p->d_col = nullptr;
            p->col_cap = 0;
            CUDA_TRY(cudaMalloc(&p->d_col, sizeof(int) * (size_t(edges) + 4)), "CsrProblem cudaMalloc d_column_indices");
            p->col_cap = size_t(edges) + 4;
        }
        // Row offsets padded with ROW_PAD entries: a bottom-up step stages 132
        // offsets (whole 16-byte units) with one bulk copy.
        if (p->row_cap < size_t(nodes) + 1 + ROW_PAD) {
            cudaFree(p->d_row_offsets);
            p->d_row_offsets = nullptr;
            p->row_cap = 0;
            CUDA_TRY(cudaMalloc(&p->d_row_offsets, sizeof(int) * (size_t(nodes) + 1 + ROW_PAD)),
                     "CsrProblem cudaMalloc d_row_offsets");
            p->row_cap = size_t(nodes) + 1 + ROW_PAD;
        }
        // The uploads are ordered on the problem's stream, ahead of the device
        // CSR check below (a plain cudaMemcpy from pageable memory may return
        // before its DMA lands, and the problem's stream does not wait for it).
        cudaStream_t s = problem_stream(p);
        CUDA_TRY(cudaMemsetAsync(p->d_col + edges, 0, 4 * sizeof(int), s), "cudaMemset column padding");
        CUDA_TRY(cudaMemsetAsync(p->d_row_offsets + nodes + 1, 0, ROW_PAD * sizeof(int), s),
                 "cudaMemset row-offset padding");
        if (edges)
            CUDA_TRY(cudaMemcpyAsync(p->d_col, h_col, sizeof(int) * size_t(edges), cudaMemcpyHostToDevice, s),
                     "CsrProblem cudaMemcpy d_column_indices");
        CUDA_TRY(cudaMemcpyAsync(p->d_row_offsets, h_row, sizeof(int) * (size_t(nodes) + 1), cudaMemcpyHostToDevice,
                                 s),
                 "CsrProblem cudaMemcpy d_row_offsets");
    }
    if ((rc = device_check_csr(p, h_row, h_col))) {
        free_problem_device(p);
        p->nodes = p->edges = 0;
        return rc;
    }
    return B40C_SUCCESS;
}

static int problem_reset(b40c_problem *p, int frontier_type, double queue_sizing, bool sync) {
    if (!p || !p->d_row_offsets) return set_error(B40C_ERR_ILLEGAL_STATE, "Reset before FromHostProblem");
    if (frontier_type < B40C_VERTEX_FRONTIERS || frontier_type > B40C_MIXED_FRONTIERS)
        return set_error(B40C_ERR_INVALID_VALUE, "Reset: frontier type %d not provided", frontier_type);
    if (!(queue_sizing > 0.0)) queue_sizing = 1.3;  // test_bfs.cu:802 default
    CUDA_TRY(cudaSetDevice(p->device), "cudaSetDevice");
    cudaStream_t s = problem_stream(p);
    // With two label buffers every Reset moves to the other one; a side copy
    // still reading it (ExtractResultsAsync two searches ago) finishes first.
    if (p->label_buffers == 2) p->use_alt = !p->use_alt;
    int *&labels = p->use_alt ? p->d_labels_alt : p->d_labels;
    size_t &labels_cap = p->use_alt ? p->labels_alt_cap : p->labels_cap;
    if (!labels) {
        CUDA_TRY(cudaMalloc(&labels, sizeof(int) * size_t(p->nodes)), "CsrProblem cudaMalloc d_labels");
        labels_cap = size_t(p->nodes);
    }
    if (p->label_buffers == 2 && p->copied[p->use_alt ? 1 : 0])
        CUDA_TRY(cudaStreamWaitEvent(s, p->copied[p->use_alt ? 1 : 0], 0), "wait for the label copy");
    // ceil(nodes / 8) bytes as the reference (csr_problem.cuh:581-583), rounded to whole words.
    p->mask_bytes = size_t((p->nodes + 31) / 32) * 4;
    if (!p->d_mask) {
        // padded so that a bottom-up step's 16-byte bulk copy of its 4 words stays inside
        CUDA_TRY(cudaMalloc(&p->d_mask, p->mask_bytes + MASK_PAD_BYTES), "CsrProblem cudaMalloc d_visited_mask");
        CUDA_TRY(cudaMemsetAsync(reinterpret_cast<char *>(p->d_mask) + p->mask_bytes, 0, MASK_PAD_BYTES, s),
                 "visited-mask padding");
        p->mask_cap = p->mask_bytes + MASK_PAD_BYTES;
    }
    long long n = p->nodes, m = p->edges;
    long long want[2] = {0, 0}, wpred[2] = {0, 0};
    // Queue sizes by frontier type (csr_problem.cuh:600-641).  Exact bitmask
    // culling bounds a vertex frontier by n and an edge frontier by m, so a
    // sizing of 1.0 never overflows; smaller factors can, and then the search
    // reports cudaErrorInvalidConfiguration as the reference does.
    auto sized = [&](long long base) {
        long long q = (long long)(double(base) * queue_sizing);
        return std::max(q, 1ll);
    };
    switch (frontier_type) {
    case B40C_VERTEX_FRONTIERS:
        want[0] = want[1] = sized(n);
        break;
    case B40C_EDGE_FRONTIERS:
        want[0] = want[1] = sized(std::max(m, n));
        if (p->mark_pred) wpred[0] = wpred[1] = want[0];
        break;
    case B40C_MIXED_FRONTIERS:
        want[0] = sized(n);
        want[1] = sized(std::max(m, n));
        if (p->mark_pred) wpred[1] = want[1];
        break;
    }
    for (int i = 0; i < 2; i++) {
        if (p->queue_elems[i] < want[i]) {
            cudaStreamSynchronize(s);
            cudaFree(p->d_queue[i]);
            p->d_queue[i] = nullptr;
            p->queue_elems[i] = 0;
            CUDA_TRY(cudaMalloc(&p->d_queue[i], sizeof(int) * size_t(want[i])),
                     "CsrProblem cudaMalloc frontier_queues.d_keys");
            p->queue_elems[i] = want[i];
        }
        if (p->pred_elems[i] < wpred[i]) {
            cudaStreamSynchronize(s);
            cudaFree(p->d_pred[i]);
            p->d_pred[i] = nullptr;
            p->pred_elems[i] = 0;
            CUDA_TRY(cudaMalloc(&p->d_pred[i], sizeof(int) * size_t(wpred[i])),
                     "CsrProblem cudaMalloc frontier_queues.d_values");
            p->pred_elems[i] = wpred[i];
        }
    }
    // labels := -1, visited mask := 0 (csr_problem.cuh:719-745).
    CUDA_TRY(launch_reset_state(labels, p->nodes, p->d_mask, (long long)(p->mask_bytes / 4), s),
             "labels and visited mask initialisation");
    p->reset_once = true;
    if (sync) CUDA_TRY(cudaStreamSynchronize(s), "Reset");
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_reset(b40c_problem_t *p, int frontier_type, double queue_sizing) {
    clear_error();
    return problem_reset(p, frontier_type, queue_sizing, true);
}

extern "C" int b40c_problem_reset_async(b40c_problem_t *p, int frontier_type, double queue_sizing) {
    clear_error();
    return problem_reset(p, frontier_type, queue_sizing, false);
}

// Enqueues the copy of the current labels to h_labels: on the problem's
// stream, or with two label buffers on the side stream behind the problem
// stream's work so far (the next Reset and search then overlap it).
static int enqueue_extract(b40c_problem *p, int *h_labels) {
    if (!p || !h_labels) return set_error(B40C_ERR_INVALID_VALUE, "ExtractResults: NULL argument");
    int *labels = cur_labels(p);
    if (!labels) return set_error(B40C_ERR_ILLEGAL_STATE, "ExtractResults before Reset");
    const size_t bytes = sizeof(int) * size_t(p->nodes);
    if (p->label_buffers == 2) {
        CUDA_TRY(cudaEventRecord(p->after_search, problem_stream(p)), "cudaEventRecord");
        CUDA_TRY(cudaStreamWaitEvent(p->copy_stream, p->after_search, 0), "cudaStreamWaitEvent");
        CUDA_TRY(cudaMemcpyAsync(h_labels, labels, bytes, cudaMemcpyDeviceToHost, p->copy_stream),
                 "CsrProblem cudaMemcpyAsync d_labels");
        CUDA_TRY(cudaEventRecord(p->copied[p->use_alt ? 1 : 0], p->copy_stream), "cudaEventRecord");
    } else {
        CUDA_TRY(cudaMemcpyAsync(h_labels, labels, bytes, cudaMemcpyDeviceToHost, problem_stream(p)),
                 "CsrProblem cudaMemcpyAsync d_labels");
    }
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_extract_results(b40c_problem_t *p, int *h_labels) {
    clear_error();
    int rc = enqueue_extract(p, h_labels);
    if (rc) return rc;
    if (p->label_buffers == 2) CUDA_TRY(cudaEventSynchronize(p->copied[p->use_alt ? 1 : 0]), "ExtractResults");
    else CUDA_TRY(cudaStreamSynchronize(problem_stream(p)), "ExtractResults");
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_from_host_ids64(b40c_problem_t *p, int stream_from_host, int nodes, int edges,
                                            const long long *h_col, const int *h_row, int num_gpus) {
    clear_error();
    if (!p || nodes <= 0 || edges < 0 || !h_row || (edges > 0 && !h_col))
        return set_error(B40C_ERR_INVALID_VALUE, "FromHostProblem: invalid arguments");
    if (stream_from_host)
        return set_error(B40C_ERR_NOT_SUPPORTED,
                         "FromHostProblem: 8-byte vertex ids are narrowed to the device's int32 layout, which "
                         "stream_from_host cannot map");
    // Every id of a graph whose sizes are int (SizeT) fits in int32: narrow
    // on several host threads, rejecting ids outside [0, nodes).
    std::vector<int> col(size_t(edges) + 1);
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<long long> bad(nt, -1);
    std::vector<std::thread> pool;
    const long long chunk = (edges + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        pool.emplace_back([&, t] {
            const long long lo = std::min<long long>(edges, t * chunk), hi = std::min<long long>(edges, lo + chunk);
            for (long long k = lo; k < hi; k++) {
                const long long v = h_col[k];
                if (v < 0 || v >= nodes) {
                    bad[t] = k;
                    break;
                }
                col[size_t(k)] = int(v);
            }
        });
    }
    for (auto &th : pool) th.join();
    for (unsigned t = 0; t < nt; t++)
        if (bad[t] >= 0)
            return set_error(B40C_ERR_INVALID_VALUE, "CSR column index %lld at edge %lld outside [0, %d)",
                             h_col[bad[t]], bad[t], nodes);
    return b40c_problem_from_host(p, 0, nodes, edges, col.data(), h_row, num_gpus);
}

extern "C" int b40c_problem_extract_results_ids64(b40c_problem_t *p, long long *h_labels) {
    clear_error();
    if (!p || !h_labels) return set_error(B40C_ERR_INVALID_VALUE, "ExtractResults: NULL argument");
    if (!cur_labels(p)) return set_error(B40C_ERR_ILLEGAL_STATE, "ExtractResults before Reset");
    std::vector<int> tmp(size_t(p->nodes));
    int rc = b40c_problem_extract_results(p, tmp.data());
    if (rc) return rc;
    for (size_t i = 0; i < tmp.size(); i++) h_labels[i] = tmp[i];
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_extract_results_async(b40c_problem_t *p, int *h_labels) {
    clear_error();
    return enqueue_extract(p, h_labels);
}

extern "C" int b40c_problem_set_label_buffers(b40c_problem_t *p, int count) {
    clear_error();
    if (!p || (count != 1 && count != 2))
        return set_error(B40C_ERR_INVALID_VALUE, "set_label_buffers: count must be 1 or 2");
    CUDA_TRY(cudaSetDevice(p->device), "cudaSetDevice");
    sync_problem(p);
    if (count == 2 && !p->copy_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking), "label copy stream");
        CUDA_TRY(cudaEventCreateWithFlags(&p->after_search, cudaEventDisableTiming), "cudaEventCreate");
        for (cudaEvent_t &ev : p->copied) CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
    }
    if (count == 1 && p->use_alt && p->d_labels_alt) {
        // Keep the current labels readable: move them into the buffer that stays.
        if (!p->d_labels) {
            CUDA_TRY(cudaMalloc(&p->d_labels, sizeof(int) * size_t(p->nodes)), "CsrProblem cudaMalloc d_labels");
            p->labels_cap = size_t(p->nodes);
        }
        CUDA_TRY(cudaMemcpy(p->d_labels, p->d_labels_alt, sizeof(int) * size_t(p->nodes), cudaMemcpyDeviceToDevice),
                 "label buffer copy");
        p->use_alt = false;
    }
    if (count == 1) {
        p->use_alt = false;
        cudaFree(p->d_labels_alt);
        p->d_labels_alt = nullptr;
        p->labels_alt_cap = 0;
    }
    p->label_buffers = count;
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_sync(b40c_problem_t *p) {
    clear_error();
    if (!p) return set_error(B40C_ERR_INVALID_VALUE, "NULL problem");
    CUDA_TRY(cudaSetDevice(p->device), "cudaSetDevice");
    CUDA_TRY(cudaStreamSynchronize(problem_stream(p)), "problem stream");
    if (p->copy_stream) CUDA_TRY(cudaStreamSynchronize(p->copy_stream), "label copy stream");
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_info(b40c_problem_t *p, int64_t *nodes, int64_t *edges, void **d_row_offsets,
                                 void **d_column_indices, void **d_labels, void **d_visited_mask) {
    clear_error();
    if (!p) return set_error(B40C_ERR_INVALID_VALUE, "NULL problem");
    if (nodes) *nodes = p->nodes;
    if (edges) *edges = p->edges;
    if (d_row_offsets) *d_row_offsets = p->d_row_offsets;
    if (d_column_indices) *d_column_indices = p->d_col;
    if (d_labels) *d_labels = cur_labels(p);
    if (d_visited_mask) *d_visited_mask = p->d_mask;
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_device(b40c_problem_t *p, int *device) {
    clear_error();
    if (!p || !device) return set_error(B40C_ERR_INVALID_VALUE, "NULL argument");
    *device = p->device;
    return B40C_SUCCESS;
}

extern "C" int b40c_problem_set_stream(b40c_problem_t *p, void *stream) {
    clear_error();
    if (!p) return set_error(B40C_ERR_INVALID_VALUE, "NULL problem");
    p->stream = (cudaStream_t)stream;
    return B40C_SUCCESS;
}

// ---- Enactors ---------------------------------------------------------------------------

extern "C" int b40c_enactor_create(int strategy, int instrument, int debug, b40c_enactor_t **out) {
    clear_error();
    if (!out) return set_error(B40C_ERR_INVALID_VALUE, "NULL out");
    if (strategy < B40C_EXPAND_CONTRACT || strategy > B40C_HYBRID)
        return set_error(B40C_ERR_INVALID_VALUE, "unknown strategy %d", strategy);
    b40c_enactor *e = new (std::nothrow) b40c_enactor();
    if (!e) return set_error(B40C_ERR_MEMORY_ALLOCATION, "enactor allocation");
    e->strategy = strategy;
    // Measured defaults: expand-contract and contract-expand run 512-thread
    // CTAs (best for both on R-MAT scale 22 and on the lattices); two-phase
    // and the hybrid run 256-thread CTAs (best on R-MAT scale 22).
    // Expand-contract gathers lists of 128+ edges with warps, the others lists
    // of 64+, and expand-contract switches direction with the published
    // alpha = 14, beta = 24 (Beamer, Asanovic and Patterson, SC 2012).
    if (strategy == B40C_EXPAND_CONTRACT) {
        e->threads = 512;
        e->warp_th = 128;
        e->do_alpha = 14;
        e->do_beta = 24;
    } else if (strategy == B40C_CONTRACT_EXPAND) {
        e->threads = 512;
    }
    e->instrument = instrument != 0;
    e->debug = debug != 0;
    cudaError_t ce = cudaGetDevice(&e->device);
    if (!ce) ce = cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking);
    if (!ce) ce = cudaEventCreate(&e->ev0);
    if (!ce) ce = cudaEventCreate(&e->ev1);
    if (ce) {
        if (e->ev0) cudaEventDestroy(e->ev0);
        if (e->own_stream) cudaStreamDestroy(e->own_stream);
        delete e;
        return cuda_fail(ce, "enactor creation");
    }
    *out = e;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_destroy(b40c_enactor_t *e) {
    clear_error();
    if (!e) return B40C_SUCCESS;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(enactor_stream(e));
    for (auto &g : e->lg) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    cudaFree(e->d_ctr);
    cudaFree(e->d_chunks[0]);
    cudaFree(e->d_chunks[1]);
    cudaFree(e->d_wchunks[0]);
    cudaFree(e->d_wchunks[1]);
    cudaFree(e->d_levels);
    cudaFree(e->d_busy);
    if (e->h_ctr) cudaFreeHost(e->h_ctr);
    cudaEventDestroy(e->ev0);
    cudaEventDestroy(e->ev1);
    if (e->own_stream) cudaStreamDestroy(e->own_stream);
    delete e;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_frontier_type(b40c_enactor_t *e, int *ft) {
    clear_error();
    if (!e || !ft) return set_error(B40C_ERR_INVALID_VALUE, "NULL argument");
    // EnactorBase(frontier_type): expand-contract uses O(n) vertex queues
    // (enactor_expand_contract.cuh), the others O(m) edge queues
    // (enactor_contract_expand.cuh:207, enactor_two_phase.cuh:222).
    *ft = e->strategy == B40C_EXPAND_CONTRACT ? B40C_VERTEX_FRONTIERS : B40C_EDGE_FRONTIERS;
    return B40C_SUCCESS;
}

extern "C" int b40c_enact_search(b40c_enactor_t *e, b40c_problem_t *p, int src, int max_grid_size, int variant) {
    clear_error();
    int rc = enqueue_search(e, p, src, max_grid_size, variant);
    if (rc) {
        if (e) cudaStreamSynchronize(enactor_stream(e));
        return rc;
    }
    rc = finish_search(e);
    if (!rc) {
        // Later problem-stream work (ExtractResults) must see the labels.
        cudaStream_t ps = problem_stream(p);
        if (ps != enactor_stream(e)) cudaStreamSynchronize(enactor_stream(e));
    }
    return rc;
}

extern "C" int b40c_enact_search_async(b40c_enactor_t *e, b40c_problem_t *p, int src, int max_grid_size,
                                       int variant) {
    clear_error();
    int rc = enqueue_search(e, p, src, max_grid_size, variant);
    if (rc) return rc;
    // Order later problem-stream work (reset, extract) after the search.
    cudaStream_t ps = problem_stream(p), s = enactor_stream(e);
    if (ps != s) {
        cudaEvent_t dep;
        CUDA_TRY(cudaEventCreateWithFlags(&dep, cudaEventDisableTiming), "cudaEventCreate");
        cudaEventRecord(dep, s);
        cudaStreamWaitEvent(ps, dep, 0);
        cudaEventDestroy(dep);
    }
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_sync(b40c_enactor_t *e) {
    clear_error();
    if (!e) return set_error(B40C_ERR_INVALID_VALUE, "NULL enactor");
    if (!e->h_ctr) return B40C_SUCCESS;
    return finish_search(e);
}

extern "C" int b40c_enactor_get_statistics(b40c_enactor_t *e, long long *total_queued, int *search_depth,
                                           double *avg_duty) {
    clear_error();
    if (!e) return set_error(B40C_ERR_INVALID_VALUE, "NULL enactor");
    if (!e->have_stats && e->h_ctr) {
        int rc = finish_search(e);
        if (rc) return rc;
    }
    // GetStatistics: search_depth = iteration - 1 (enactor_contract_expand.cuh:245).
    if (total_queued) *total_queued = e->instrument ? e->last_total_queued : 0;
    if (search_depth) *search_depth = e->last_iteration - 1;
    if (avg_duty) *avg_duty = e->instrument ? e->last_duty : 0.0;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_last_elapsed_ms(b40c_enactor_t *e, float *ms) {
    clear_error();
    if (!e || !ms) return set_error(B40C_ERR_INVALID_VALUE, "NULL argument");
    *ms = e->last_ms;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_set_stream(b40c_enactor_t *e, void *stream) {
    clear_error();
    if (!e) return set_error(B40C_ERR_INVALID_VALUE, "NULL enactor");
    e->stream = (cudaStream_t)stream;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_set_policy(b40c_enactor_t *e, int cta_threads, int warp_th, int cta_th,
                                       int cull_flags) {
    clear_error();
    if (!e) return set_error(B40C_ERR_INVALID_VALUE, "NULL enactor");
    if (cta_threads && cta_threads != 128 && cta_threads != 256 && cta_threads != 512)
        return set_error(B40C_ERR_INVALID_VALUE, "cta_threads must be 128, 256 or 512");
    if (warp_th < 0 || cta_th < 0 || cull_flags < -1 || cull_flags > 3)
        return set_error(B40C_ERR_INVALID_VALUE, "invalid policy field");
    if (cta_threads) e->threads = cta_threads;
    if (warp_th) e->warp_th = warp_th;
    if (cta_th) e->cta_th = cta_th;
    if (cull_flags >= 0) e->cull_flags = unsigned(cull_flags);
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_set_level_log(b40c_enactor_t *e, int enable) {
    clear_error();
    if (!e) return set_error(B40C_ERR_INVALID_VALUE, "NULL enactor");
    e->log_levels = enable != 0;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_level_log(b40c_enactor_t *e, int max_records, int64_t *t_start_ns, int *frontier,
                                      int *chunks, int *wchunks, int *bottom_up, int *count) {
    clear_error();
    if (!e || !count || max_records < 0) return set_error(B40C_ERR_INVALID_VALUE, "invalid argument");
    *count = 0;
    if (!e->log_levels || !e->d_levels) return set_error(B40C_ERR_ILLEGAL_STATE, "level log not enabled");
    if (e->h_ctr && !e->have_stats) {
        int rc = finish_search(e);
        if (rc) return rc;
    }
    std::vector<LevelRecord> h(LEVEL_LOG_CAP);
    CUDA_TRY(cudaMemcpy(h.data(), e->d_levels, sizeof(LevelRecord) * LEVEL_LOG_CAP, cudaMemcpyDeviceToHost),
             "level log copy");
    // Records run up to the end-of-search marker (no frontier, no chunks).
    int n = 0;
    while (n < LEVEL_LOG_CAP && h[n].t_start != 0) {
        n++;
        if (h[n - 1].frontier == 0u && h[n - 1].chunks == 0u && h[n - 1].wchunks == 0u) break;
    }
    n = std::min(n, max_records);
    for (int i = 0; i < n; i++) {
        if (t_start_ns) t_start_ns[i] = (int64_t)h[i].t_start;
        if (frontier) frontier[i] = (int)h[i].frontier;
        if (chunks) chunks[i] = (int)h[i].chunks;
        if (wchunks) wchunks[i] = (int)h[i].wchunks;
        if (bottom_up) bottom_up[i] = (int)h[i].bottom_up;
    }
    *count = n;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_level_times(b40c_enactor_t *e, int max_records, int64_t *t_start_ns,
                                        int64_t *t_work_end_ns, int *count) {
    clear_error();
    if (!e || !count || max_records < 0) return set_error(B40C_ERR_INVALID_VALUE, "invalid argument");
    *count = 0;
    if (!e->log_levels || !e->d_levels) return set_error(B40C_ERR_ILLEGAL_STATE, "level log not enabled");
    if (e->h_ctr && !e->have_stats) {
        int rc = finish_search(e);
        if (rc) return rc;
    }
    std::vector<LevelRecord> h(LEVEL_LOG_CAP);
    CUDA_TRY(cudaMemcpy(h.data(), e->d_levels, sizeof(LevelRecord) * LEVEL_LOG_CAP, cudaMemcpyDeviceToHost),
             "level log copy");
    int n = 0;
    while (n < LEVEL_LOG_CAP && h[n].t_start != 0) {
        n++;
        if (h[n - 1].frontier == 0u && h[n - 1].chunks == 0u && h[n - 1].wchunks == 0u) break;
    }
    n = std::min(n, max_records);
    for (int i = 0; i < n; i++) {
        if (t_start_ns) t_start_ns[i] = (int64_t)h[i].t_start;
        if (t_work_end_ns) t_work_end_ns[i] = (int64_t)h[i].t_work_end;
    }
    *count = n;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_set_direction_optimizing(b40c_enactor_t *e, int alpha, int beta) {
    clear_error();
    if (!e || alpha < 0 || beta < 0 || (alpha > 0 && beta == 0))
        return set_error(B40C_ERR_INVALID_VALUE, "direction switch: alpha >= 0, and beta >= 1 when alpha > 0");
    if (alpha > 0 && e->strategy != B40C_EXPAND_CONTRACT)
        return set_error(B40C_ERR_NOT_SUPPORTED, "bottom-up levels exist for the expand-contract strategy only");
    e->do_alpha = unsigned(alpha);
    e->do_beta = unsigned(beta);
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_set_wait_limit_us(b40c_enactor_t *e, long long us) {
    clear_error();
    if (!e || us <= 0) return set_error(B40C_ERR_INVALID_VALUE, "invalid wait limit");
    e->wait_ns = (unsigned long long)us * 1000ull;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_set_bottom_up_staging(b40c_enactor_t *e, int enable) {
    clear_error();
    if (!e) return set_error(B40C_ERR_INVALID_VALUE, "NULL enactor");
    e->stage_bu = enable != 0;
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_set_narrow_levels(b40c_enactor_t *e, int team_ctas, int max_frontier,
                                              int grid_frontier) {
    clear_error();
    if (!e) return set_error(B40C_ERR_INVALID_VALUE, "NULL enactor");
    if (team_ctas < 0 || team_ctas > 16 || max_frontier < 0 || grid_frontier < 0)
        return set_error(B40C_ERR_INVALID_VALUE,
                         "narrow levels: team_ctas in [0, 16], max_frontier >= 0, grid_frontier >= 0");
    e->narrow_team = team_ctas;
    e->narrow_max = unsigned(max_frontier);
    e->flat_max = unsigned(grid_frontier);
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_narrow_team(b40c_enactor_t *e, int *team) {
    clear_error();
    if (!e || !team) return set_error(B40C_ERR_INVALID_VALUE, "NULL argument");
    *team = 0;
    if (e->narrow_team == 0) return B40C_SUCCESS;
    CUDA_TRY(cudaSetDevice(e->device), "cudaSetDevice");
    const KernelConfig kc{e->strategy, e->threads, false};
    CUDA_TRY(narrow_team_limit(kc, e->narrow_team, team), "cluster occupancy query");
    return B40C_SUCCESS;
}

extern "C" int b40c_enactor_set_l2_persistence(b40c_enactor_t *e, int what) {
    clear_error();
    if (!e || what < 0 || what > 2) return set_error(B40C_ERR_INVALID_VALUE, "L2 persistence: what is 0, 1 or 2");
    e->l2_persist = what;
    return B40C_SUCCESS;
}

// ---- failure detection ------------------------------------------------------------------

extern "C" int b40c_debug_barrier_timeout(int grid_size, long long wait_limit_us) {
    clear_error();
    if (grid_size < 1 || grid_size > 4096 || wait_limit_us <= 0 || wait_limit_us > 10000000)
        return set_error(B40C_ERR_INVALID_VALUE, "invalid probe arguments");
    unsigned err = 0;
    cudaError_t e = run_barrier_timeout_probe(grid_size, (unsigned long long)wait_limit_us * 1000ull, &err);
    if (e) return cuda_fail(e, "barrier timeout probe");
    return translate_device_error(err);
}
