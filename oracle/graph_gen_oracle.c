/*
 * graph_gen_oracle.c -- seeded benchmark inputs, restated for the checker.
 *
 * TEST INFRASTRUCTURE ONLY.  The CPU legs of the benchmark (the reference's
 * own BFS timed on the host cores) and the tests build their R-MAT inputs and
 * draw their sources here, so that they never load the product library.  The
 * product's generators (back40computing_b200/csrc/graph_gen.cpp,
 * b40c_graph_rmat and b40c_graph_sample_sources) define the workload; this is
 * a second, independent statement of the same definition, and
 * tests/test_oracle.py pins the two together by the sha256 of the CSR arrays
 * and by the sampled sources.
 *
 * The workload definition (not the reference's GTgraph builder, which draws
 * with rand(), 1-based ids and per-level noise, b40c/graph/builder/rmat.cuh:
 * 83-116, :167-169):
 *   - edge e of m = edge_factor << scale draws its own splitmix64 stream
 *     (Steele, Lea and Flood, OOPSLA 2014) seeded from (seed, e): one value is
 *     discarded, then one value per level picks a quadrant with probabilities
 *     a, b, c, 1 - a - b - c, from the top bit of the vertex ids down
 *     (Graph500-style recursive R-MAT, 0-based, no permutation);
 *   - self-loops are dropped, duplicates kept; an undirected graph lists
 *     every forward edge (u, v) first and then every reversed edge (v, u),
 *     and the CSR keeps that list order inside each row (a stable sort by
 *     row, as CsrGraph::FromCoo, b40c/graph/csr_graph.cuh:108-152).
 *   - sources: splitmix64 draws modulo the vertex count, kept when the vertex
 *     has at least one edge.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t sm64_next(uint64_t *state) {
    uint64_t z = (*state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double unit_interval(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

typedef struct {
    int scale;
    double a, ab, abc;
    uint64_t seed;
    int64_t lo, hi;
    int *u, *v;
} rmat_job_t;

static void *rmat_worker(void *arg) {
    rmat_job_t *j = (rmat_job_t *)arg;
    int64_t e;
    for (e = j->lo; e < j->hi; e++) {
        uint64_t st = j->seed * 0xD1B54A32D192ED03ull ^ ((uint64_t)e * 0x9E3779B97F4A7C15ull);
        int64_t u = 0, v = 0;
        int lvl;
        sm64_next(&st);
        for (lvl = j->scale - 1; lvl >= 0; lvl--) {
            double r = unit_interval(sm64_next(&st));
            int ub = r >= j->ab, vb = (r >= j->a && r < j->ab) || r >= j->abc;
            u |= (int64_t)ub << lvl;
            v |= (int64_t)vb << lvl;
        }
        j->u[e] = (int)u;
        j->v[e] = (int)v;
    }
    return NULL;
}

/* R-MAT CSR as defined above.  *row_offsets (nodes + 1) and *column_indices
 * (edges, plus 4 zero entries of padding) are malloc'd; free them with
 * oracle_free.  Returns 0, or -1 on bad arguments / allocation failure. */
int oracle_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int undirected,
                int threads, int64_t *nodes_out, int64_t *edges_out, int **row_offsets, int **column_indices) {
    int64_t nodes, m, list_len, k, edges = 0;
    int *u, *v, *row, *col;
    int64_t *cursor;
    pthread_t tid[256];
    rmat_job_t job[256];
    int t;
    if (scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 + 1e-12) return -1;
    nodes = (int64_t)1 << scale;
    m = (int64_t)edge_factor << scale;
    list_len = undirected ? 2 * m : m;
    if (list_len > INT32_MAX - 8) return -1;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    u = (int *)malloc(sizeof(int) * (size_t)m);
    v = (int *)malloc(sizeof(int) * (size_t)m);
    row = (int *)calloc((size_t)nodes + 1, sizeof(int));
    cursor = (int64_t *)calloc((size_t)nodes + 1, sizeof(int64_t));
    if (!u || !v || !row || !cursor) {
        free(u);
        free(v);
        free(row);
        free(cursor);
        return -1;
    }
    for (t = 0; t < threads; t++) {
        job[t].scale = scale;
        job[t].a = a;
        job[t].ab = a + b;
        job[t].abc = a + b + c;
        job[t].seed = seed;
        job[t].lo = m * t / threads;
        job[t].hi = m * (t + 1) / threads;
        job[t].u = u;
        job[t].v = v;
        pthread_create(&tid[t], NULL, rmat_worker, &job[t]);
    }
    for (t = 0; t < threads; t++) pthread_join(tid[t], NULL);
    /* stable counting sort of the edge list by row */
    for (k = 0; k < list_len; k++) {
        int64_t e = k < m ? k : k - m;
        if (u[e] == v[e]) continue;
        cursor[k < m ? u[e] : v[e]]++;
        edges++;
    }
    {
        int64_t run = 0, r;
        for (r = 0; r < nodes; r++) {
            int64_t cnt = cursor[r];
            row[r] = (int)run;
            cursor[r] = run;
            run += cnt;
        }
        row[nodes] = (int)run;
    }
    col = (int *)malloc(sizeof(int) * (size_t)(edges + 4));
    if (!col) {
        free(u);
        free(v);
        free(row);
        free(cursor);
        return -1;
    }
    for (k = 0; k < list_len; k++) {
        int64_t e = k < m ? k : k - m;
        if (u[e] == v[e]) continue;
        if (k < m) col[cursor[u[e]]++] = v[e];
        else col[cursor[v[e]]++] = u[e];
    }
    memset(col + edges, 0, 4 * sizeof(int));
    free(u);
    free(v);
    free(cursor);
    *nodes_out = nodes;
    *edges_out = edges;
    *row_offsets = row;
    *column_indices = col;
    return 0;
}

/* num_sources vertices of degree > 0 drawn from the seeded stream defined
 * above.  Returns 0, or -1 when the graph has no edges. */
int oracle_sample_sources(int64_t nodes, const int *row_offsets, int num_sources, uint64_t seed, int *sources) {
    uint64_t st = seed * 0x8CB92BA72F3D8DD7ull + 0x2545F4914F6CDD1Dull;
    int64_t w;
    int i, any = 0;
    for (w = 0; w < nodes && !any; w++) any = row_offsets[w + 1] > row_offsets[w];
    if (!any) return -1;
    for (i = 0; i < num_sources; i++) {
        for (;;) {
            int64_t x = (int64_t)(sm64_next(&st) % (uint64_t)nodes);
            if (row_offsets[x + 1] > row_offsets[x]) {
                sources[i] = (int)x;
                break;
            }
        }
    }
    return 0;
}

void oracle_free(void *p) { free(p); }
