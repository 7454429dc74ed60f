/*
 * b40c/graph/bfs/enactors.hpp -- drop-in for back40computing's
 * b40c/graph/bfs/enactor_{contract_expand,expand_contract,two_phase,hybrid}.cuh:
 * the Enactor classes with EnactSearch / EnactFusedSearch /
 * EnactIterativeSearch / GetStatistics / GetFrontierType, header-only C++
 * over the C ABI of libb40c_bfs.so.  A test_bfs.cu-style caller
 * (test/bfs/test_bfs.cu:600-756) compiles against these unchanged.
 */
#pragma once

#include <cuda_runtime_api.h>

#include "b40c/graph/bfs/csr_problem.hpp"
#include "b40c_bfs.h"

namespace b40c {
namespace graph {
namespace bfs {

/* Shared enactor machinery (enactor_base.cuh:55-126). */
template <int STRATEGY, bool INSTRUMENT>
class EnactorCommon {
  protected:
    b40c_enactor_t *handle;

  public:
    bool DEBUG;

    explicit EnactorCommon(bool DEBUG = false) : handle(0), DEBUG(DEBUG) {
        b40c_enactor_create(STRATEGY, INSTRUMENT ? 1 : 0, DEBUG ? 1 : 0, &handle);
    }
    virtual ~EnactorCommon() { b40c_enactor_destroy(handle); }

    /* enactor_base.cuh:72 */
    FrontierType GetFrontierType() {
        int ft = 0;
        b40c_enactor_frontier_type(handle, &ft);
        return (FrontierType)ft;
    }

    /* EnactSearch(problem, src, max_grid_size): the strategy's default variant
     * (the persistent fused kernel). */
    template <class CsrProblem>
    cudaError_t EnactSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, int max_grid_size = 0) {
        return (cudaError_t)b40c_enact_search(handle, csr_problem.handle, (int)src, max_grid_size,
                                              B40C_VARIANT_DEFAULT);
    }
    /* One persistent launch for all levels (e.g. enactor_contract_expand.cuh:259-407). */
    template <class CsrProblem>
    cudaError_t EnactFusedSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, int max_grid_size = 0) {
        return (cudaError_t)b40c_enact_search(handle, csr_problem.handle, (int)src, max_grid_size,
                                              B40C_VARIANT_FUSED);
    }
    /* Per-level kernels; the level loop runs on the device in a CUDA graph
     * (e.g. enactor_two_phase.cuh:416-614). */
    template <class CsrProblem>
    cudaError_t EnactIterativeSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src,
                                     int max_grid_size = 0) {
        return (cudaError_t)b40c_enact_search(handle, csr_problem.handle, (int)src, max_grid_size,
                                              B40C_VARIANT_ITERATIVE);
    }

    /* enactor_contract_expand.cuh:237-250: search_depth = iteration - 1. */
    template <typename VertexId>
    void GetStatistics(long long &total_queued, VertexId &search_depth, double &avg_duty) {
        int depth = 0;
        b40c_enactor_get_statistics(handle, &total_queued, &depth, &avg_duty);
        search_depth = (VertexId)depth;
    }

    /* KernelPolicy knobs (kernel_policy.cuh:61-87) as runtime settings. */
    cudaError_t SetPolicy(int cta_threads, int warp_gather_threshold, int cta_gather_threshold, int cull_flags = -1) {
        return (cudaError_t)b40c_enactor_set_policy(handle, cta_threads, warp_gather_threshold,
                                                    cta_gather_threshold, cull_flags);
    }
    /* Options with no counterpart in the reference (b40c_bfs.h): the
     * expand-contract direction switch (alpha = 0: top-down only), and the
     * narrow levels of high-diameter searches (team_ctas = 0: off). */
    cudaError_t SetDirectionOptimizing(int alpha, int beta) {
        return (cudaError_t)b40c_enactor_set_direction_optimizing(handle, alpha, beta);
    }
    cudaError_t SetNarrowLevels(int team_ctas, int max_frontier, int grid_frontier) {
        return (cudaError_t)b40c_enactor_set_narrow_levels(handle, team_ctas, max_frontier, grid_frontier);
    }

  private:
    EnactorCommon(const EnactorCommon &);
    EnactorCommon &operator=(const EnactorCommon &);
};

/* enactor_expand_contract.cuh:59-526 */
template <bool INSTRUMENT>
class EnactorExpandContract : public EnactorCommon<B40C_EXPAND_CONTRACT, INSTRUMENT> {
  public:
    explicit EnactorExpandContract(bool DEBUG = false) : EnactorCommon<B40C_EXPAND_CONTRACT, INSTRUMENT>(DEBUG) {}
};

/* enactor_contract_expand.cuh:61-598 */
template <bool INSTRUMENT>
class EnactorContractExpand : public EnactorCommon<B40C_CONTRACT_EXPAND, INSTRUMENT> {
  public:
    explicit EnactorContractExpand(bool DEBUG = false) : EnactorCommon<B40C_CONTRACT_EXPAND, INSTRUMENT>(DEBUG) {}
};

/* enactor_two_phase.cuh:68-766 */
template <bool INSTRUMENT>
class EnactorTwoPhase : public EnactorCommon<B40C_TWO_PHASE, INSTRUMENT> {
  public:
    explicit EnactorTwoPhase(bool DEBUG = false) : EnactorCommon<B40C_TWO_PHASE, INSTRUMENT>(DEBUG) {}
};

/* enactor_hybrid.cuh:64-758: contract-expand levels while the edge frontier is
 * small, two-phase levels while it is large (one persistent launch here).  The
 * reference class offers only EnactSearch; EnactFusedSearch and
 * EnactIterativeSearch run the same search. */
template <bool INSTRUMENT>
class EnactorHybrid : public EnactorCommon<B40C_HYBRID, INSTRUMENT> {
  public:
    explicit EnactorHybrid(bool DEBUG = false) : EnactorCommon<B40C_HYBRID, INSTRUMENT>(DEBUG) {}
};

}  // namespace bfs
}  // namespace graph
}  // namespace b40c
