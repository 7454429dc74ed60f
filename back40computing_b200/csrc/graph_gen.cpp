// Host CSR graph builders: the inputs of the BFS path.
//
// These play the role of b40c's builders (b40c/graph/builder/grid2d.cuh:53-114,
// grid3d.cuh:53-129, rmat.cuh:127-206, csr_graph.cuh:108-152).  Two deliberate
// differences from the reference builders:
//   * lattices get no self-loops unless asked (the reference appends one per
//     vertex, grid2d.cuh:102-104), because the benchmark graphs are defined
//     without them; with self_loops=1 the CSR is identical to the reference's;
//   * R-MAT uses a counter-based RNG (splitmix64 per edge and level) and the
//     Graph500 0-based quadrant recursion without per-level noise, so a graph
//     is a pure function of (scale, edge_factor, a, b, c, seed) and can be
//     generated in parallel.  The reference's GTgraph variant uses rand(),
//     1-based ids and +-5% noise per level (rmat.cuh:83-116, :167-169).
// Row order follows CsrGraph::FromCoo: a stable sort of the COO list by row,
// where an undirected list is [forward edges..., reversed edges...]
// (rmat.cuh:180-185), so rows keep generation order.

#include "b40c_bfs.h"
#include "host_common.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace b40c_b200 {

static inline uint64_t splitmix64(uint64_t &state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline double to_unit(uint64_t x) {  // [0, 1)
    return double(x >> 11) * (1.0 / 9007199254740992.0);
}

static int host_threads() {
    unsigned t = std::thread::hardware_concurrency();
    if (t == 0) t = 1;
    if (t > 64) t = 64;
    return int(t);
}

template <class F>
static void parallel_for_chunks(int64_t total, int threads, F fn) {
    if (threads <= 1 || total < (1 << 16)) {
        fn(0, int64_t(0), total);
        return;
    }
    std::vector<std::thread> pool;
    int64_t chunk = (total + threads - 1) / threads;
    for (int t = 0; t < threads; t++) {
        int64_t lo = std::min<int64_t>(total, t * chunk);
        int64_t hi = std::min<int64_t>(total, lo + chunk);
        pool.emplace_back([=] { fn(t, lo, hi); });
    }
    for (auto &th : pool) th.join();
}

static int alloc_csr(int64_t nodes, int64_t edges, b40c_csr_t *out) {
    out->nodes = nodes;
    out->edges = edges;
    // Column array padded by 4 entries so 16-byte vector loads of a list tail
    // stay inside the allocation when the array is uploaded verbatim.
    out->row_offsets = (int *)std::malloc(sizeof(int) * size_t(nodes + 1));
    out->column_indices = (int *)std::malloc(sizeof(int) * size_t(edges + 4));
    if (!out->row_offsets || !out->column_indices) {
        std::free(out->row_offsets);
        std::free(out->column_indices);
        out->row_offsets = nullptr;
        out->column_indices = nullptr;
        return set_error(B40C_ERR_MEMORY_ALLOCATION, "host allocation of %lld-edge CSR failed",
                         (long long)edges);
    }
    std::memset(out->column_indices + edges, 0, 4 * sizeof(int));
    return B40C_SUCCESS;
}

// Stable counting sort of a directed edge list into CSR.  Entry k of the list
// is produced by get(k, &row, &col) and is skipped when get returns false.
// Each thread owns a contiguous slice of the list; per-thread row counts give
// every thread its write cursor inside each row, which keeps list order.
template <class Get>
static int build_csr_stable(int64_t nodes, int64_t list_len, Get get, b40c_csr_t *out) {
    if (nodes <= 0 || nodes > INT32_MAX - 1)
        return set_error(B40C_ERR_INVALID_VALUE, "node count %lld out of range", (long long)nodes);
    int threads = host_threads();
    if (list_len < (1 << 16)) threads = 1;
    // Bound the per-thread count arrays to ~1 GiB.
    while (threads > 1 && double(threads) * double(nodes) * 8.0 > double(1ull << 30)) threads /= 2;

    std::vector<std::vector<int64_t>> cnt(threads, std::vector<int64_t>(size_t(nodes), 0));
    int64_t chunk = (list_len + threads - 1) / threads;
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; t++) {
            pool.emplace_back([&, t] {
                int64_t lo = std::min<int64_t>(list_len, t * chunk);
                int64_t hi = std::min<int64_t>(list_len, lo + chunk);
                int64_t *c = cnt[t].data();
                for (int64_t k = lo; k < hi; k++) {
                    int r, col;
                    if (get(k, r, col)) c[r]++;
                }
            });
        }
        for (auto &th : pool) th.join();
    }
    // Exclusive prefix over rows; turn cnt[t][row] into thread t's cursor in row.
    int64_t total = 0;
    std::vector<int64_t> row_start(size_t(nodes) + 1);
    for (int64_t r = 0; r < nodes; r++) {
        row_start[r] = total;
        int64_t run = total;
        for (int t = 0; t < threads; t++) {
            int64_t c = cnt[t][r];
            cnt[t][r] = run;
            run += c;
        }
        total = run;
    }
    row_start[nodes] = total;
    if (total > INT32_MAX - 8)
        return set_error(B40C_ERR_INVALID_VALUE, "%lld directed edges exceed int32 SizeT",
                         (long long)total);
    int rc = alloc_csr(nodes, total, out);
    if (rc) return rc;
    for (int64_t r = 0; r <= nodes; r++) out->row_offsets[r] = int(row_start[r]);
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; t++) {
            pool.emplace_back([&, t] {
                int64_t lo = std::min<int64_t>(list_len, t * chunk);
                int64_t hi = std::min<int64_t>(list_len, lo + chunk);
                int64_t *c = cnt[t].data();
                int *col_out = out->column_indices;
                for (int64_t k = lo; k < hi; k++) {
                    int r, col;
                    if (get(k, r, col)) col_out[c[r]++] = col;
                }
            });
        }
        for (auto &th : pool) th.join();
    }
    return B40C_SUCCESS;
}

}  // namespace b40c_b200

using namespace b40c_b200;

extern "C" int b40c_graph_grid2d(int width, int self_loops, b40c_csr_t *out) {
    if (!out || width <= 0 || int64_t(width) * width > INT32_MAX / 8)
        return set_error(B40C_ERR_INVALID_VALUE, "grid2d: invalid width %d", width);
    int64_t w = width, nodes = w * w;
    int64_t edges = 0;
    for (int64_t j = 0; j < w; j++)
        for (int64_t k = 0; k < w; k++)
            edges += (k > 0) + (k + 1 < w) + (j > 0) + (j + 1 < w) + (self_loops ? 1 : 0);
    int rc = alloc_csr(nodes, edges, out);
    if (rc) return rc;
    int64_t total = 0;
    int *col = out->column_indices;
    // Neighbour order of builder/grid2d.cuh:72-104: left, right, up, down, self.
    for (int64_t j = 0; j < w; j++) {
        for (int64_t k = 0; k < w; k++) {
            int64_t me = j * w + k;
            out->row_offsets[me] = int(total);
            if (k - 1 >= 0) col[total++] = int(me - 1);
            if (k + 1 < w) col[total++] = int(me + 1);
            if (j - 1 >= 0) col[total++] = int(me - w);
            if (j + 1 < w) col[total++] = int(me + w);
            if (self_loops) col[total++] = int(me);
        }
    }
    out->row_offsets[nodes] = int(total);
    return B40C_SUCCESS;
}

extern "C" int b40c_graph_grid3d(int width, int self_loops, b40c_csr_t *out) {
    if (!out || width <= 0 || int64_t(width) * width * width > INT32_MAX / 8)
        return set_error(B40C_ERR_INVALID_VALUE, "grid3d: invalid width %d", width);
    int64_t w = width, plane = w * w, nodes = plane * w;
    int64_t edges = 3 * 2 * (w - 1) * plane + (self_loops ? nodes : 0);
    int rc = alloc_csr(nodes, edges, out);
    if (rc) return rc;
    // Neighbour order of builder/grid3d.cuh:73-118: k-1, k+1, j-1, j+1, i-1, i+1, self.
    int threads = host_threads();
    std::vector<int64_t> slab_start(size_t(w) + 1, 0);
    for (int64_t i = 0; i < w; i++) {
        int64_t per_slab = 0;
        for (int64_t j = 0; j < w; j++)
            for (int64_t k = 0; k < w; k++)
                per_slab += (k > 0) + (k + 1 < w) + (j > 0) + (j + 1 < w) + (i > 0) + (i + 1 < w) +
                            (self_loops ? 1 : 0);
        slab_start[i + 1] = slab_start[i] + per_slab;
    }
    if (slab_start[w] != edges)
        return set_error(B40C_ERR_INVALID_VALUE, "grid3d: edge count mismatch");
    int *col = out->column_indices;
    int *ro = out->row_offsets;
    parallel_for_chunks(w, threads, [&](int, int64_t ilo, int64_t ihi) {
        for (int64_t i = ilo; i < ihi; i++) {
            int64_t total = slab_start[i];
            for (int64_t j = 0; j < w; j++) {
                for (int64_t k = 0; k < w; k++) {
                    int64_t me = i * plane + j * w + k;
                    ro[me] = int(total);
                    if (k - 1 >= 0) col[total++] = int(me - 1);
                    if (k + 1 < w) col[total++] = int(me + 1);
                    if (j - 1 >= 0) col[total++] = int(me - w);
                    if (j + 1 < w) col[total++] = int(me + w);
                    if (i - 1 >= 0) col[total++] = int(me - plane);
                    if (i + 1 < w) col[total++] = int(me + plane);
                    if (self_loops) col[total++] = int(me);
                }
            }
        }
    });
    ro[nodes] = int(edges);
    return B40C_SUCCESS;
}

extern "C" int b40c_graph_rmat(int scale, int edge_factor, double a, double b, double c,
                               uint64_t seed, int undirected, b40c_csr_t *out) {
    if (!out || scale < 1 || scale > 30 || edge_factor < 1)
        return set_error(B40C_ERR_INVALID_VALUE, "rmat: invalid scale %d / edge factor %d", scale,
                         edge_factor);
    double d = 1.0 - a - b - c;
    if (a < 0 || b < 0 || c < 0 || d < -1e-12)
        return set_error(B40C_ERR_INVALID_VALUE, "rmat: invalid quadrant probabilities");
    int64_t nodes = int64_t(1) << scale;
    int64_t m = int64_t(edge_factor) << scale;
    if ((undirected ? 2 * m : m) > INT32_MAX - 8)
        return set_error(B40C_ERR_INVALID_VALUE, "rmat: %lld edges exceed int32 SizeT",
                         (long long)(undirected ? 2 * m : m));
    std::vector<int> U((size_t)m), V((size_t)m);
    const double ab = a + b, abc = a + b + c;
    parallel_for_chunks(m, host_threads(), [&](int, int64_t lo, int64_t hi) {
        for (int64_t e = lo; e < hi; e++) {
            // Independent stream per edge: a function of (seed, e) only.
            uint64_t st = seed * 0xD1B54A32D192ED03ull ^ (uint64_t(e) * 0x9E3779B97F4A7C15ull);
            splitmix64(st);
            int64_t u = 0, v = 0;
            for (int lvl = scale - 1; lvl >= 0; lvl--) {
                double r = to_unit(splitmix64(st));
                int ub, vb;
                if (r < a) { ub = 0; vb = 0; }
                else if (r < ab) { ub = 0; vb = 1; }
                else if (r < abc) { ub = 1; vb = 0; }
                else { ub = 1; vb = 1; }
                u |= int64_t(ub) << lvl;
                v |= int64_t(vb) << lvl;
            }
            U[e] = int(u);
            V[e] = int(v);
        }
    });
    int64_t list_len = undirected ? 2 * m : m;
    return build_csr_stable(
        nodes, list_len,
        [&](int64_t k, int &r, int &col) -> bool {
            int64_t e = k < m ? k : k - m;
            int u = U[e], v = V[e];
            if (u == v) return false;  // self-loops removed
            if (k < m) { r = u; col = v; }
            else { r = v; col = u; }
            return true;
        },
        out);
}

extern "C" int b40c_graph_erdos_renyi(int nodes, double p, uint64_t seed, b40c_csr_t *out) {
    if (!out || nodes <= 1 || !(p > 0.0) || p >= 1.0)
        return set_error(B40C_ERR_INVALID_VALUE, "erdos_renyi: invalid n=%d p=%g", nodes, p);
    // Batagelj-Brandes geometric skipping over the pairs (v, w), w < v.
    std::vector<int> U, V;
    U.reserve(size_t(double(nodes) * (nodes - 1) * 0.5 * p * 1.1) + 16);
    V.reserve(U.capacity());
    uint64_t st = seed * 0xA24BAED4963EE407ull + 0x9FB21C651E98DF25ull;
    const double lq = std::log(1.0 - p);
    int64_t v = 1, w = -1;
    while (v < nodes) {
        double r = to_unit(splitmix64(st));
        w += 1 + int64_t(std::floor(std::log(1.0 - r) / lq));
        while (w >= v && v < nodes) {
            w -= v;
            v++;
        }
        if (v < nodes) {
            U.push_back(int(v));
            V.push_back(int(w));
        }
    }
    int64_t m = int64_t(U.size());
    if (2 * m > INT32_MAX - 8)
        return set_error(B40C_ERR_INVALID_VALUE, "erdos_renyi: too many edges");
    return build_csr_stable(
        nodes, 2 * m,
        [&](int64_t k, int &r, int &col) -> bool {
            int64_t e = k < m ? k : k - m;
            if (k < m) { r = U[e]; col = V[e]; }
            else { r = V[e]; col = U[e]; }
            return true;
        },
        out);
}

extern "C" int b40c_graph_from_coo(int nodes, int64_t num_edges, const int *rows, const int *cols,
                                   b40c_csr_t *out) {
    if (!out || nodes <= 0 || num_edges < 0 || (num_edges > 0 && (!rows || !cols)))
        return set_error(B40C_ERR_INVALID_VALUE, "from_coo: invalid arguments");
    for (int64_t k = 0; k < num_edges; k++) {
        if (rows[k] < 0 || rows[k] >= nodes || cols[k] < 0 || cols[k] >= nodes)
            return set_error(B40C_ERR_INVALID_VALUE, "from_coo: edge %lld (%d,%d) out of range",
                             (long long)k, rows[k], cols[k]);
    }
    return build_csr_stable(
        nodes, num_edges,
        [&](int64_t k, int &r, int &col) -> bool {
            r = rows[k];
            col = cols[k];
            return true;
        },
        out);
}

extern "C" int b40c_csr_free(b40c_csr_t *csr) {
    if (!csr) return set_error(B40C_ERR_INVALID_VALUE, "csr_free: NULL");
    std::free(csr->row_offsets);
    std::free(csr->column_indices);
    csr->row_offsets = nullptr;
    csr->column_indices = nullptr;
    csr->nodes = csr->edges = 0;
    return B40C_SUCCESS;
}

extern "C" int b40c_graph_sample_sources(const b40c_csr_t *csr, int num_sources, uint64_t seed,
                                         int *sources) {
    if (!csr || !csr->row_offsets || num_sources < 0 || (num_sources > 0 && !sources))
        return set_error(B40C_ERR_INVALID_VALUE, "sample_sources: invalid arguments");
    int64_t n = csr->nodes;
    bool any = false;
    for (int64_t v = 0; v < n && !any; v++) any = csr->row_offsets[v + 1] > csr->row_offsets[v];
    if (!any) return set_error(B40C_ERR_INVALID_VALUE, "sample_sources: graph has no edges");
    uint64_t st = seed * 0x8CB92BA72F3D8DD7ull + 0x2545F4914F6CDD1Dull;
    for (int i = 0; i < num_sources; i++) {
        for (;;) {
            int64_t v = int64_t(splitmix64(st) % uint64_t(n));
            if (csr->row_offsets[v + 1] > csr->row_offsets[v]) {
                sources[i] = int(v);
                break;
            }
        }
    }
    return B40C_SUCCESS;
}
