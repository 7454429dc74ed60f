/*
 * bfs_oracle.c -- CPU oracle for the BFS path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (libb40c_bfs.so, the
 * back40computing_b200 package) links, loads or calls this file; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg do, as the checker.
 *
 * It restates, in plain C, the reference's serial CPU BFS and validators from
 * back40computing's test driver:
 *   oracle_bfs                 <- SimpleReferenceBfs, test/bfs/test_bfs.cu:503-578
 *   oracle_compare_labels      <- CompareResults, test/b40c_test_util.h:303-339
 *   oracle_check_predecessors  <- DisplayStats (MARK_PREDECESSORS branch),
 *                                 test/bfs/test_bfs.cu:379-440
 *   oracle_visit_stats         <- DisplayStats nodes/edges visited, :354-367
 * Parity is pinned: tests/golden holds labels produced by the reference's own
 * SimpleReferenceBfs (compiled from its sources by oracle/Makefile into
 * oracle/_ref), and the CPU test suite checks this restatement against them.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Labels: -1 unvisited, depth otherwise (source 0).  FIFO over an array in
 * place of std::deque; same visit order, same labels.  Returns the
 * reference's search_depth: deepest label + 1 (test_bfs.cu:541-557). */
int64_t oracle_bfs(int64_t nodes, const int *row_offsets, const int *column_indices, int src,
                   int *labels) {
    int64_t i, head = 0, tail = 0;
    int search_depth = 0;
    int *frontier;
    if (nodes <= 0 || src < 0 || src >= nodes) return -1;
    frontier = (int *)malloc(sizeof(int) * (size_t)nodes);
    if (!frontier) return -2;
    for (i = 0; i < nodes; i++) labels[i] = -1;
    labels[src] = 0;
    frontier[tail++] = src;
    while (head < tail) {
        int node = frontier[head++];
        int neighbor_dist = labels[node] + 1;
        int e, begin = row_offsets[node], end = row_offsets[node + 1];
        for (e = begin; e < end; e++) {
            int neighbor = column_indices[e];
            if (labels[neighbor] == -1) {
                labels[neighbor] = neighbor_dist;
                if (search_depth < neighbor_dist) search_depth = neighbor_dist;
                frontier[tail++] = neighbor;
            }
        }
    }
    free(frontier);
    return (int64_t)search_depth + 1;
}

/* Index of the first differing label, or -1 when identical. */
int64_t oracle_compare_labels(int64_t nodes, const int *computed, const int *reference) {
    int64_t i;
    for (i = 0; i < nodes; i++)
        if (computed[i] != reference[i]) return i;
    return -1;
}

/* Validity of a predecessor labelling against reference depths.  Returns -1
 * when every node passes, else the first failing node; *reason gets
 * 1 = parentless node with positive depth, 2 = parent depth != depth - 1,
 * 3 = parent is not adjacent to the node. */
int64_t oracle_check_predecessors(int64_t nodes, const int *row_offsets, const int *column_indices,
                                  const int *preds, const int *ref_depths, int *reason) {
    int64_t node;
    for (node = 0; node < nodes; node++) {
        int parent = preds[node];
        int node_dist = ref_depths[node];
        int e, found = 0;
        if (parent < 0) {
            if (node_dist > 0) {
                if (reason) *reason = 1;
                return node;
            }
            continue;
        }
        if (parent >= nodes || ref_depths[parent] + 1 != node_dist) {
            if (reason) *reason = 2;
            return node;
        }
        for (e = row_offsets[parent]; e < row_offsets[parent + 1]; e++) {
            if (column_indices[e] == node) {
                found = 1;
                break;
            }
        }
        if (!found) {
            if (reason) *reason = 3;
            return node;
        }
    }
    if (reason) *reason = 0;
    return -1;
}

/* nodes_visited = #labels > -1; edges_visited = sum of their degrees. */
void oracle_visit_stats(int64_t nodes, const int *row_offsets, const int *labels,
                        int64_t *nodes_visited, int64_t *edges_visited) {
    int64_t i, nv = 0, ev = 0;
    for (i = 0; i < nodes; i++) {
        if (labels[i] > -1) {
            nv++;
            ev += row_offsets[i + 1] - row_offsets[i];
        }
    }
    if (nodes_visited) *nodes_visited = nv;
    if (edges_visited) *edges_visited = ev;
}

/* ---- independent searches on several host threads (CPU baseline) ---- */
typedef struct {
    int64_t nodes;
    const int *row_offsets, *column_indices;
    const int *sources;
    int num_sources;
    int stride, first;
    int64_t *edges_visited;
    int *labels; /* per-thread scratch of nodes labels */
} oracle_job_t;

static void *oracle_worker(void *arg) {
    oracle_job_t *job = (oracle_job_t *)arg;
    int s;
    for (s = job->first; s < job->num_sources; s += job->stride) {
        int64_t ev = 0;
        oracle_bfs(job->nodes, job->row_offsets, job->column_indices, job->sources[s], job->labels);
        oracle_visit_stats(job->nodes, job->row_offsets, job->labels, NULL, &ev);
        job->edges_visited[s] = ev;
    }
    return NULL;
}

/* Runs one search per source over threads host threads (sources round-robin).
 * edges_visited[s] receives each search's edges_visited.  Returns 0 or -1. */
int oracle_bfs_many(int64_t nodes, const int *row_offsets, const int *column_indices,
                    const int *sources, int num_sources, int threads, int64_t *edges_visited) {
    pthread_t tid[256];
    oracle_job_t job[256];
    int t, rc = 0;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    for (t = 0; t < threads; t++) {
        job[t].nodes = nodes;
        job[t].row_offsets = row_offsets;
        job[t].column_indices = column_indices;
        job[t].sources = sources;
        job[t].num_sources = num_sources;
        job[t].stride = threads;
        job[t].first = t;
        job[t].edges_visited = edges_visited;
        job[t].labels = (int *)malloc(sizeof(int) * (size_t)nodes);
        if (!job[t].labels) rc = -1;
    }
    if (rc == 0) {
        for (t = 0; t < threads; t++) pthread_create(&tid[t], NULL, oracle_worker, &job[t]);
        for (t = 0; t < threads; t++) pthread_join(tid[t], NULL);
    }
    for (t = 0; t < threads; t++) free(job[t].labels);
    return rc;
}

/* ---- reference labels of many sources at once (parity checks) ---- */
typedef struct {
    int64_t nodes;
    const int *row_offsets, *column_indices;
    const int *sources;
    int num_sources;
    int stride, first;
    int *labels; /* num_sources x nodes */
    int64_t *depths;
} oracle_labels_job_t;

static void *oracle_labels_worker(void *arg) {
    oracle_labels_job_t *job = (oracle_labels_job_t *)arg;
    int s;
    for (s = job->first; s < job->num_sources; s += job->stride)
        job->depths[s] = oracle_bfs(job->nodes, job->row_offsets, job->column_indices, job->sources[s],
                                    job->labels + (size_t)s * (size_t)job->nodes);
    return NULL;
}

/* SimpleReferenceBfs from every source, spread over threads host threads:
 * labels[s * nodes + v] receives source s's labels and depths[s] its
 * search_depth (as oracle_bfs).  Returns 0. */
int oracle_bfs_many_labels(int64_t nodes, const int *row_offsets, const int *column_indices,
                           const int *sources, int num_sources, int threads, int *labels, int64_t *depths) {
    pthread_t tid[256];
    oracle_labels_job_t job[256];
    int t;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if (threads > num_sources) threads = num_sources > 0 ? num_sources : 1;
    for (t = 0; t < threads; t++) {
        job[t].nodes = nodes;
        job[t].row_offsets = row_offsets;
        job[t].column_indices = column_indices;
        job[t].sources = sources;
        job[t].num_sources = num_sources;
        job[t].stride = threads;
        job[t].first = t;
        job[t].labels = labels;
        job[t].depths = depths;
    }
    for (t = 0; t < threads; t++) pthread_create(&tid[t], NULL, oracle_labels_worker, &job[t]);
    for (t = 0; t < threads; t++) pthread_join(tid[t], NULL);
    return 0;
}

