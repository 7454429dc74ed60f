"""B200 (sm_100a) breadth-first search with the b40c::graph::bfs API of back40computing.

The compute path is libb40c_bfs.so (hand-written CUDA kernels behind a C ABI,
include/b40c_bfs.h); this package is its Python host side.
"""
from .bfs import (  # noqa: F401
    BfsError,
    CsrProblem,
    EnactorContractExpand,
    EnactorExpandContract,
    EnactorHybrid,
    EnactorTwoPhase,
    FrontierType,
    Strategy,
    Variant,
    check,
    make_enactor,
)
from .graphs import (CsrGraph, erdos_renyi, from_coo, grid2d, grid3d, read_dimacs, read_market,  # noqa: F401
                     read_metis, rmat)
