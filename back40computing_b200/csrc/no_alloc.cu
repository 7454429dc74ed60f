// Breadth-first search that allocates no memory: b40c_enact_search_no_alloc.
//
// Some callers cannot call cudaMalloc at search time: frameworks whose
// allocator owns every byte of the device and forbids allocation behind its
// back, and real-time loops that cannot pay for the device-wide
// synchronisation that cudaMalloc/cudaFree may imply.  For them this entry
// point runs the fused expand-contract search over a CSR and a label array
// the caller already holds on the device.  The scratch memory the search
// needs besides those (search counters, visited bitmask, the two frontier
// queues and the CTA and warp chunk tables) is carved from one file-scope
// device array of a fixed size, NOALLOC_SCRATCH_BYTES, which every GPU that
// loads this library holds until the process exits.
//
// Host code cannot use the array's name as a device address (on the host it
// names a host-side stand-in), so the first call in each CUDA context looks
// up the array's device address with cudaGetSymbolAddress and keeps it for
// that context; a new context (after cudaDeviceReset, or a context the caller
// made current) gets its own lookup.
//
// Every call shares the one array, and a call leaves its contents behind: each
// call therefore clears the counters and the visited bitmask (they must start
// at zero) and sets the caller's labels to -1; the queues and chunk tables are
// written before they are read and need no clearing.  Two calls whose work
// overlaps on the GPU (different streams, or different host threads, on the
// same device) race on the array and corrupt each other's results.

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "b40c_bfs.h"
#include "bfs_kernels.cuh"
#include "host_common.h"

using namespace b40c_b200;

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(32) << 20;  // 32 MiB per device
constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_WARP_TH = 128;   // expand-contract default warp gather threshold
constexpr int NOALLOC_CTA_TH = 1024;   // default CTA gather threshold
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mutex;
void *g_noalloc_base[NOALLOC_MAX_DEVICES] = {};
unsigned long long g_noalloc_ctx[NOALLOC_MAX_DEVICES] = {};  // context id the address belongs to

size_t round256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of the pieces carved from the scratch array for a graph.
struct ScratchLayout {
    size_t ctr, mask, queue[2], chunks[2], wchunks[2], total;
    size_t mask_bytes;
    long long chunk_cap, wchunk_cap;
};

// Same capacities as the enactor's own buffers: a vertex frontier holds each
// vertex at most once (exact bitmask cull), and a neighbour list of len edges
// placed in CH-edge chunks takes at most len / CH + 2 entries, for at most
// edges / threshold lists per level.
ScratchLayout layout_for(long long nodes, long long edges) {
    ScratchLayout L{};
    L.chunk_cap = edges / chunk_edges<NOALLOC_THREADS>() + 2 * (edges / NOALLOC_CTA_TH) + 64;
    L.wchunk_cap = edges / WARP_CHUNK + 2 * (edges / NOALLOC_WARP_TH) + 64;
    L.mask_bytes = size_t((nodes + 31) / 32) * sizeof(unsigned);
    size_t off = 0;
    L.ctr = off;
    off += round256(sizeof(Counters));
    L.mask = off;
    off += round256(L.mask_bytes);
    for (int i = 0; i < 2; i++) {
        L.queue[i] = off;
        off += round256(size_t(nodes) * sizeof(int));
    }
    for (int i = 0; i < 2; i++) {
        L.chunks[i] = off;
        off += round256(size_t(L.chunk_cap) * sizeof(int4));
    }
    for (int i = 0; i < 2; i++) {
        L.wchunks[i] = off;
        off += round256(size_t(L.wchunk_cap) * sizeof(int4));
    }
    L.total = off;
    return L;
}

int cuda_fail(cudaError_t e, const char *what) {
    return set_error(int(e), "no-alloc search: %s failed (CUDA error %d: %s)", what, int(e), cudaGetErrorString(e));
}
#define NA_TRY(call, what)                                  \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, what);  \
    } while (0)

// Id of the calling thread's current CUDA context (driver entry points found
// through the runtime, so the library links no libcuda); 0 when unknown.
unsigned long long current_context_id() {
    typedef CUresult (*GetCurrentFn)(CUcontext *);
    typedef CUresult (*GetIdFn)(CUcontext, unsigned long long *);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetIdFn>(f);
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS)
        return id;
    return 0;
}

// Device address of the scratch array in the current context.  It is looked
// up once per device and context (symbol addresses belong to a context, and a
// reset device gets a new one); when the context id cannot be read, it is
// looked up on every call (the lookup allocates nothing).
int scratch_base(int device, unsigned char **base) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    const unsigned long long ctx = current_context_id();
    if (!g_noalloc_base[device] || ctx == 0 || g_noalloc_ctx[device] != ctx) {
        void *p = nullptr;
        NA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress of the scratch array");
        g_noalloc_base[device] = p;
        g_noalloc_ctx[device] = ctx;
    }
    *base = static_cast<unsigned char *>(g_noalloc_base[device]);
    return B40C_SUCCESS;
}

int device_error(unsigned err) {
    if (err & ERR_BAD_VERTEX)
        return set_error(B40C_ERR_INVALID_VALUE, "no-alloc search: column index outside [0, nodes)");
    if (err & ERR_BARRIER_TIMEOUT)
        return set_error(B40C_ERR_LAUNCH_TIMEOUT, "no-alloc search: grid barrier wait exceeded its limit");
    if (err & ERR_LEVEL_LIMIT)
        return set_error(B40C_ERR_LAUNCH_TIMEOUT, "no-alloc search: level loop passed nodes + 2 levels");
    if (err & ERR_OVERFLOW)
        return set_error(B40C_ERR_INVALID_CONFIGURATION, "no-alloc search: frontier queue overflow");
    return B40C_SUCCESS;
}

}  // namespace

extern "C" int b40c_enact_search_no_alloc(int nodes, int edges, const int *d_row_offsets,
                                          const int *d_column_indices, int src, int *d_labels,
                                          int *search_depth, void *stream) {
    clear_error();
    if (nodes <= 0 || edges < 0)
        return set_error(B40C_ERR_INVALID_VALUE, "no-alloc search: nodes must be > 0 and edges >= 0");
    const ScratchLayout L = layout_for(nodes, edges);
    if (L.total > NOALLOC_SCRATCH_BYTES)
        return set_error(B40C_ERR_INVALID_VALUE,
                         "no-alloc search: a graph of %d vertices and %d edges needs %zu bytes of scratch, more "
                         "than the %zu bytes of the library's static scratch array",
                         nodes, edges, L.total, NOALLOC_SCRATCH_BYTES);
    if (!d_row_offsets || !d_labels || (edges > 0 && !d_column_indices))
        return set_error(B40C_ERR_INVALID_VALUE, "no-alloc search: NULL row offsets, column indices or labels");
    if (src < 0 || src >= nodes)
        return set_error(B40C_ERR_INVALID_VALUE, "no-alloc search: source %d outside [0, %d)", src, nodes);
    int device = 0;
    NA_TRY(cudaGetDevice(&device), "cudaGetDevice");
    if (device < 0 || device >= NOALLOC_MAX_DEVICES)
        return set_error(B40C_ERR_INVALID_VALUE, "no-alloc search: device ordinal %d not supported", device);
    unsigned char *base = nullptr;
    int rc = scratch_base(device, &base);
    if (rc) return rc;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BfsParams bp{};
    bp.row_offsets = d_row_offsets;
    bp.col = d_column_indices;
    bp.labels = d_labels;
    bp.mask = reinterpret_cast<unsigned *>(base + L.mask);
    for (int i = 0; i < 2; i++) {
        bp.queue[i] = reinterpret_cast<int *>(base + L.queue[i]);
        bp.pred_queue[i] = nullptr;
        bp.chunks[i] = reinterpret_cast<int4 *>(base + L.chunks[i]);
        bp.wchunks[i] = reinterpret_cast<int4 *>(base + L.wchunks[i]);
    }
    bp.levels = nullptr;
    bp.level_cap = 0;
    bp.ctr = reinterpret_cast<Counters *>(base + L.ctr);
    bp.wait_ns = 5000000000ull;
    bp.cond_handle = 0;
    bp.qcap = nodes;
    bp.chunk_cap = int(L.chunk_cap);
    bp.wchunk_cap = int(L.wchunk_cap);
    // The caller's column array has no padding: 16-byte loads stop at the
    // last whole group of four, and none are used if it is not 16-byte aligned.
    bp.vec_end = (reinterpret_cast<uintptr_t>(d_column_indices) & 15u) ? 0 : (edges & ~3);
    bp.nodes = nodes;
    bp.src = src;
    bp.warp_th = NOALLOC_WARP_TH;
    bp.cta_th = NOALLOC_CTA_TH;
    bp.cull_flags = CULL_HISTORY;
    bp.stream_col = 1;  // column loads keep their evict_first L2 policy
    const KernelConfig kc{STRATEGY_EXPAND_CONTRACT, NOALLOC_THREADS, false};

    // What must start at zero (counters, sticky error word included, and the
    // visited bitmask) is cleared; labels start at -1 as Reset leaves them.
    NA_TRY(cudaMemsetAsync(bp.ctr, 0, sizeof(Counters), s), "counters clear");
    NA_TRY(cudaMemsetAsync(bp.mask, 0, L.mask_bytes, s), "visited mask clear");
    NA_TRY(cudaMemsetAsync(d_labels, 0xff, sizeof(int) * size_t(nodes), s), "labels clear");
    NA_TRY(launch_search_init(bp, kc, s), "search init kernel launch");
    int grid = 0;
    NA_TRY(fused_grid_limit(kc, &grid), "occupancy query");
    NA_TRY(launch_fused(bp, kc, grid, s), "cooperative launch of the fused BFS kernel");
    Counters h;  // pageable host copy: the library holds no pinned buffer for this call
    NA_TRY(cudaMemcpyAsync(&h, bp.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s), "counters copy");
    NA_TRY(cudaStreamSynchronize(s), "no-alloc BFS search");
    if ((rc = device_error(h.error | h.sticky))) return rc;
    // GetStatistics: search_depth = iteration - 1 (enactor_contract_expand.cuh:245).
    if (search_depth) *search_depth = h.iteration - 1;
    return B40C_SUCCESS;
}
