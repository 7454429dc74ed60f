/*
 * b40c/graph/bfs/csr_problem.hpp -- drop-in for b40c/graph/bfs/csr_problem.cuh
 * of back40computing: bfs::CsrProblem and FrontierType, header-only C++ over
 * the C ABI of libb40c_bfs.so (include/b40c_bfs.h).  Only the single-GPU
 * branch is provided (num_gpus <= 1).
 */
#pragma once

#include <cuda_runtime_api.h>

#include "b40c_bfs.h"

namespace b40c {
namespace graph {
namespace bfs {

/* csr_problem.cuh:54-61 */
enum FrontierType {
    VERTEX_FRONTIERS = B40C_VERTEX_FRONTIERS,
    EDGE_FRONTIERS = B40C_EDGE_FRONTIERS,
    MIXED_FRONTIERS = B40C_MIXED_FRONTIERS,
    MULTI_GPU_FRONTIERS = B40C_MULTI_GPU_FRONTIERS,
    MULTI_GPU_VERTEX_FRONTIER_SCALE = 2,
};

/* problem_type.cuh:47-70: the type traits callers name through CsrProblem::ProblemType */
template <typename _VertexId, typename _SizeT, bool _MARK_PREDECESSORS>
struct ProblemType {
    typedef _VertexId VertexId;
    typedef _SizeT SizeT;
    typedef unsigned char VisitedMask;
    typedef unsigned char ValidFlag;
    static const bool MARK_PREDECESSORS = _MARK_PREDECESSORS;
};

/* Host-side id width of FromHostProblem / ExtractResults: 4-byte ids go to
 * the device as they are; 8-byte ids (the reference's g500 configuration,
 * VertexId = long long with int sizes) are narrowed to the device's int32
 * layout and widened on the way back. */
inline int b40c_from_host_any(b40c_problem_t *h, int sfh, int n, int m, int *col, int *row, int g) {
    return b40c_problem_from_host(h, sfh, n, m, col, row, g);
}
inline int b40c_from_host_any(b40c_problem_t *h, int sfh, int n, int m, long long *col, int *row, int g) {
    return b40c_problem_from_host_ids64(h, sfh, n, m, col, row, g);
}
inline int b40c_extract_any(b40c_problem_t *h, int *labels) { return b40c_problem_extract_results(h, labels); }
inline int b40c_extract_any(b40c_problem_t *h, long long *labels) {
    return b40c_problem_extract_results_ids64(h, labels);
}

/*
 * bfs::CsrProblem<VertexId, SizeT, MARK_PREDECESSORS> (csr_problem.cuh:68-751).
 * SizeT must be int; VertexId int, or long long as the reference's g500
 * graphs use (test/bfs/test_bfs.cu:1068-1093).  The device layout is int32
 * either way: with 8-byte ids the slice's d_column_indices / d_labels point
 * at int32 arrays.  Members that reference callers read -- nodes, edges,
 * num_gpus, and the single graph slice's device pointers -- are kept up to
 * date.
 */
template <typename _VertexId, typename _SizeT, bool MARK_PREDECESSORS>
struct CsrProblem {
    static_assert((sizeof(_VertexId) == 4 || sizeof(_VertexId) == 8) && sizeof(_SizeT) == 4,
                  "the B200 BFS takes int or long long vertex ids with int sizes");

    typedef bfs::ProblemType<_VertexId, _SizeT, MARK_PREDECESSORS> ProblemType;
    typedef typename ProblemType::VertexId VertexId;
    typedef typename ProblemType::SizeT SizeT;
    typedef typename ProblemType::VisitedMask VisitedMask;
    typedef typename ProblemType::ValidFlag ValidFlag;

    /* GraphSlice (csr_problem.cuh:99-173), device pointers of GPU 0 */
    struct GraphSlice {
        int gpu;
        VertexId *d_column_indices;
        SizeT *d_row_offsets;
        VertexId *d_labels;
        VisitedMask *d_visited_mask;
        VertexId nodes;
        SizeT edges;
    };

    int num_gpus;
    SizeT nodes;
    SizeT edges;
    GraphSlice slice;
    GraphSlice *graph_slices[1];
    b40c_problem_t *handle;

    CsrProblem() : num_gpus(0), nodes(0), edges(0), handle(0) {
        slice = GraphSlice();
        graph_slices[0] = &slice;
        b40c_problem_create(MARK_PREDECESSORS ? 1 : 0, &handle);
    }
    virtual ~CsrProblem() { b40c_problem_destroy(handle); }

    /* csr_problem.cuh:328-403 */
    cudaError_t FromHostProblem(bool stream_from_host, SizeT nodes, SizeT edges, VertexId *h_column_indices,
                                SizeT *h_row_offsets, int num_gpus) {
        int rc = b40c_from_host_any(handle, stream_from_host ? 1 : 0, (int)nodes, (int)edges, h_column_indices,
                                    (int *)h_row_offsets, num_gpus);
        if (rc == 0) {
            this->nodes = nodes;
            this->edges = edges;
            this->num_gpus = 1;
            refresh();
        }
        return (cudaError_t)rc;
    }

    /* csr_problem.cuh:547-750 */
    cudaError_t Reset(FrontierType frontier_type, double queue_sizing) {
        int rc = b40c_problem_reset(handle, (int)frontier_type, queue_sizing);
        if (rc == 0) refresh();
        return (cudaError_t)rc;
    }

    /* csr_problem.cuh:255-273 */
    cudaError_t ExtractResults(VertexId *h_label) {
        return (cudaError_t)b40c_extract_any(handle, h_label);
    }

    /* csr_problem.cuh:188-218 (one slice) */
    template <typename V>
    int GpuIndex(V) {
        return slice.gpu;
    }
    template <typename V>
    V GraphSliceRow(V vertex) {
        return vertex;
    }

  private:
    void refresh() {
        int64_t n = 0, m = 0;
        void *ro = 0, *ci = 0, *lb = 0, *vm = 0;
        b40c_problem_info(handle, &n, &m, &ro, &ci, &lb, &vm);
        b40c_problem_device(handle, &slice.gpu);
        slice.d_row_offsets = (SizeT *)ro;
        slice.d_column_indices = (VertexId *)ci;
        slice.d_labels = (VertexId *)lb;
        slice.d_visited_mask = (VisitedMask *)vm;
        slice.nodes = (VertexId)n;
        slice.edges = (SizeT)m;
    }
    CsrProblem(const CsrProblem &);
    CsrProblem &operator=(const CsrProblem &);
};

}  // namespace bfs
}  // namespace graph
}  // namespace b40c
