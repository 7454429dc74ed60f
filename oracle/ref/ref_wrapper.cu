/*
 * ref_wrapper.cu -- builds the reference's own CPU BFS into oracle/_ref/libref_bfs.so.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference source test/bfs/test_bfs.cu is
 * included unmodified from the read-only reference tree at build time (see
 * oracle/Makefile), with its main() renamed.  Only host code is called:
 *   ref_simple_bfs      -> SimpleReferenceBfs       (test/bfs/test_bfs.cu:503-578)
 *   ref_build_grid2d/3d -> BuildGrid2dGraph/3d      (b40c/graph/builder/grid2d.cuh:53, grid3d.cuh:53)
 *   ref_build_random    -> BuildRandomGraph         (b40c/graph/builder/random.cuh:53)
 *   ref_build_rmat      -> BuildRmatGraph           (b40c/graph/builder/rmat.cuh:127)
 *   ref_from_coo        -> CsrGraph::FromCoo        (b40c/graph/csr_graph.cuh:108)
 * Its printf output is sent to /dev/null while these run.
 */
#define main b40c_reference_test_bfs_main
#include "bfs/test_bfs.cu"
#undef main

#include <fcntl.h>
#include <unistd.h>
#include <cstdint>
#include <thread>
#include <vector>

namespace {
struct Quiet {  // silence stdout (fd 1) for the lifetime of the object
    int saved;
    Quiet() {
        fflush(stdout);
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        dup2(devnull, 1);
        close(devnull);
    }
    ~Quiet() {
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

typedef b40c::graph::CsrGraph<int, int, int> Graph;

int run_one(int nodes, int edges, int *row_offsets, int *column_indices, int src, int *labels) {
    Graph g(false);
    g.nodes = nodes;
    g.edges = edges;
    g.row_offsets = row_offsets;
    g.column_indices = column_indices;
    char name[] = "reference CPU BFS";
    Stats stats(name);
    SimpleReferenceBfs(-1, g, labels, src, stats);
    g.row_offsets = NULL;  // caller-owned: keep ~CsrGraph from freeing them
    g.column_indices = NULL;
    int depth = -1;
    for (int i = 0; i < nodes; i++)
        if (labels[i] > depth) depth = labels[i];
    return depth + 1;  // search_depth as SimpleReferenceBfs computes it
}

int export_graph(Graph &g, int64_t *nodes, int64_t *edges, int **row_offsets, int **column_indices) {
    *nodes = g.nodes;
    *edges = g.edges;
    *row_offsets = g.row_offsets;
    *column_indices = g.column_indices;
    g.row_offsets = NULL;
    g.column_indices = NULL;
    g.values = NULL;
    return 0;
}
}  // namespace

extern "C" int ref_simple_bfs(int nodes, int edges, int *row_offsets, int *column_indices, int src,
                              int *labels) {
    Quiet q;
    return run_one(nodes, edges, row_offsets, column_indices, src, labels);
}

/* Independent searches, one per source, over `threads` host threads. */
extern "C" int ref_simple_bfs_many(int nodes, int edges, int *row_offsets, int *column_indices,
                                   const int *sources, int num_sources, int threads,
                                   int64_t *edges_visited) {
    Quiet q;
    if (threads < 1) threads = 1;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) {
        pool.emplace_back([=] {
            std::vector<int> labels(nodes);
            for (int s = t; s < num_sources; s += threads) {
                run_one(nodes, edges, row_offsets, column_indices, sources[s], labels.data());
                int64_t ev = 0;
                for (int v = 0; v < nodes; v++)
                    if (labels[v] > -1) ev += row_offsets[v + 1] - row_offsets[v];
                edges_visited[s] = ev;
            }
        });
    }
    for (auto &th : pool) th.join();
    return 0;
}

extern "C" int ref_build_grid2d(int width, int64_t *nodes, int64_t *edges, int **row_offsets,
                                int **column_indices) {
    Quiet q;
    Graph g(false);
    if (b40c::graph::builder::BuildGrid2dGraph<false>(width, g)) return -1;
    return export_graph(g, nodes, edges, row_offsets, column_indices);
}

extern "C" int ref_build_grid3d(int width, int64_t *nodes, int64_t *edges, int **row_offsets,
                                int **column_indices) {
    Quiet q;
    Graph g(false);
    if (b40c::graph::builder::BuildGrid3dGraph<false>(width, g)) return -1;
    return export_graph(g, nodes, edges, row_offsets, column_indices);
}

/* srand(seed) then the reference builder (rand()-driven). */
extern "C" int ref_build_random(int nodes, int edges, int undirected, unsigned seed, int64_t *n_out,
                                int64_t *m_out, int **row_offsets, int **column_indices) {
    Quiet q;
    Graph g(false);
    srand(seed);
    if (b40c::graph::builder::BuildRandomGraph<false>(nodes, edges, g, undirected != 0)) return -1;
    return export_graph(g, n_out, m_out, row_offsets, column_indices);
}

extern "C" int ref_build_rmat(int nodes, int edges, int undirected, double a, double b, double c,
                              unsigned seed, int64_t *n_out, int64_t *m_out, int **row_offsets,
                              int **column_indices) {
    Quiet q;
    Graph g(false);
    srand(seed);
    if (b40c::graph::builder::BuildRmatGraph<false>(nodes, edges, g, undirected != 0, a, b, c))
        return -1;
    return export_graph(g, n_out, m_out, row_offsets, column_indices);
}

extern "C" int ref_from_coo(int nodes, int num_edges, const int *rows, const int *cols,
                            int64_t *n_out, int64_t *m_out, int **row_offsets, int **column_indices) {
    Quiet q;
    typedef b40c::graph::CooEdgeTuple<int, int> Tuple;
    Tuple *coo = (Tuple *)malloc(sizeof(Tuple) * (size_t)(num_edges > 0 ? num_edges : 1));
    for (int i = 0; i < num_edges; i++) {
        coo[i].row = rows[i];
        coo[i].col = cols[i];
        coo[i].val = 1;
    }
    Graph g(false);
    g.template FromCoo<false>(coo, nodes, num_edges);
    free(coo);
    return export_graph(g, n_out, m_out, row_offsets, column_indices);
}

extern "C" void ref_free(void *p) { free(p); }

/* The reference's graph-file readers (b40c/graph/builder/market.cuh,
 * metis.cuh, dimacs.cuh), for pinning this package's readers. */
extern "C" int ref_read_market(const char *path, int undirected, int64_t *n_out, int64_t *m_out, int **row_offsets,
                               int **column_indices) {
    Quiet q;
    Graph g(false);
    if (b40c::graph::builder::BuildMarketGraph<false>((char *)path, g, undirected != 0)) return -1;
    return export_graph(g, n_out, m_out, row_offsets, column_indices);
}

extern "C" int ref_read_metis(const char *path, int64_t *n_out, int64_t *m_out, int **row_offsets,
                              int **column_indices) {
    Quiet q;
    Graph g(false);
    if (b40c::graph::builder::BuildMetisGraph<false>((char *)path, g)) return -1;
    return export_graph(g, n_out, m_out, row_offsets, column_indices);
}

extern "C" int ref_read_dimacs(const char *path, int undirected, int64_t *n_out, int64_t *m_out, int **row_offsets,
                               int **column_indices) {
    Quiet q;
    Graph g(false);
    if (b40c::graph::builder::BuildDimacsGraph<false>((char *)path, g, undirected != 0, 0)) return -1;
    return export_graph(g, n_out, m_out, row_offsets, column_indices);
}
