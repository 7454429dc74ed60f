"""Python mirror of b40c::graph::bfs (back40computing), over the C ABI.

Names, argument meaning and return values follow the reference C++ API so that
callers read like test/bfs/test_bfs.cu:600-756:

    problem = CsrProblem(mark_predecessors=False)
    problem.FromHostProblem(False, nodes, edges, h_column_indices, h_row_offsets, 1)
    enactor = EnactorContractExpand()
    problem.Reset(enactor.GetFrontierType(), 1.3)
    enactor.EnactSearch(problem, src)          # -> cudaError_t value, 0 on success
    problem.ExtractResults(h_labels)
    total_queued, search_depth, avg_duty = enactor.GetStatistics()

Every method returns the cudaError_t code the reference would (0 = success);
``check(code)`` raises :class:`BfsError` with the library's message instead.
"""
from __future__ import annotations

import ctypes
from enum import IntEnum

import numpy as np

from ._lib import last_error, lib
from .graphs import CsrGraph


class FrontierType(IntEnum):
    """b40c/graph/bfs/csr_problem.cuh:54-61."""
    VERTEX_FRONTIERS = 0
    EDGE_FRONTIERS = 1
    MIXED_FRONTIERS = 2
    MULTI_GPU_FRONTIERS = 3


class Strategy(IntEnum):
    """test/bfs/test_bfs.cu:71-78."""
    EXPAND_CONTRACT = 0
    CONTRACT_EXPAND = 1
    TWO_PHASE = 2
    HYBRID = 3


class Variant(IntEnum):
    DEFAULT = 0
    FUSED = 1
    ITERATIVE = 2


# cudaError_t values the library returns
cudaSuccess = 0
cudaErrorInvalidValue = 1
cudaErrorMemoryAllocation = 2
cudaErrorInvalidConfiguration = 9
cudaErrorInvalidDeviceFunction = 98
cudaErrorIllegalState = 401
cudaErrorLaunchTimeout = 702
cudaErrorNotSupported = 801


class BfsError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{message} (cudaError_t {code})")
        self.code = code
        self.message = message


def check(code: int) -> None:
    if code:
        raise BfsError(code, last_error())


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return a.ctypes.data_as(ctypes.c_void_p)


class CsrProblem:
    """bfs::CsrProblem<int, int, MARK_PREDECESSORS> (csr_problem.cuh:68-751)."""

    def __init__(self, mark_predecessors: bool = False):
        self.MARK_PREDECESSORS = bool(mark_predecessors)
        h = ctypes.c_void_p()
        check(lib().b40c_problem_create(int(mark_predecessors), ctypes.byref(h)))
        self._h = h
        self.nodes = 0
        self.edges = 0
        self._host_refs = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().b40c_problem_destroy(h)
            except Exception:
                pass
            self._h = None

    close = __del__

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def FromHostProblem(self, stream_from_host: bool, nodes: int, edges: int, h_column_indices,
                        h_row_offsets, num_gpus: int = 1) -> int:
        """csr_problem.cuh:328-403; the host arrays stay owned by the caller."""
        col = np.ascontiguousarray(h_column_indices, dtype=np.int32)
        row = np.ascontiguousarray(h_row_offsets, dtype=np.int32)
        if row.shape[0] < nodes + 1 or col.shape[0] < edges:
            return cudaErrorInvalidValue
        rc = lib().b40c_problem_from_host(self._h, int(stream_from_host), int(nodes), int(edges),
                                          _ptr(col), _ptr(row), int(num_gpus))
        if rc == 0:
            self.nodes, self.edges = int(nodes), int(edges)
            # Mapped (stream_from_host) arrays must outlive the problem.
            self._host_refs = (col, row) if stream_from_host else None
        return rc

    def from_graph(self, g: CsrGraph, stream_from_host: bool = False) -> "CsrProblem":
        check(self.FromHostProblem(stream_from_host, g.nodes, g.edges, g.column_indices, g.row_offsets, 1))
        return self

    def Reset(self, frontier_type: int, queue_sizing: float = 1.3) -> int:
        """csr_problem.cuh:547-750 (synchronous)."""
        return lib().b40c_problem_reset(self._h, int(frontier_type), float(queue_sizing))

    def ResetAsync(self, frontier_type: int, queue_sizing: float = 1.3) -> int:
        return lib().b40c_problem_reset_async(self._h, int(frontier_type), float(queue_sizing))

    def ExtractResults(self, h_labels: np.ndarray) -> int:
        """csr_problem.cuh:255-273: copies `nodes` int32 labels into h_labels."""
        if h_labels.dtype != np.int32 or not h_labels.flags.c_contiguous or h_labels.shape[0] < self.nodes:
            return cudaErrorInvalidValue
        return lib().b40c_problem_extract_results(self._h, _ptr(h_labels))

    def ExtractResultsAsync(self, h_labels: np.ndarray) -> int:
        if h_labels.dtype != np.int32 or not h_labels.flags.c_contiguous or h_labels.shape[0] < self.nodes:
            return cudaErrorInvalidValue
        return lib().b40c_problem_extract_results_async(self._h, _ptr(h_labels))

    def labels(self) -> np.ndarray:
        out = np.empty(self.nodes, np.int32)
        check(self.ExtractResults(out))
        return out

    def device_pointers(self) -> dict:
        n, m = ctypes.c_int64(), ctypes.c_int64()
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        check(lib().b40c_problem_info(self._h, ctypes.byref(n), ctypes.byref(m), *[ctypes.byref(p) for p in ptrs]))
        return {"nodes": n.value, "edges": m.value, "d_row_offsets": ptrs[0].value,
                "d_column_indices": ptrs[1].value, "d_labels": ptrs[2].value, "d_visited_mask": ptrs[3].value}

    def set_stream(self, stream_handle: int | None) -> None:
        check(lib().b40c_problem_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    def set_label_buffers(self, count: int) -> None:
        """count = 2: Reset alternates two label arrays and ExtractResultsAsync
        copies on a side stream, overlapping the next search (no reference
        counterpart; the reference keeps one d_labels array)."""
        check(lib().b40c_problem_set_label_buffers(self._h, int(count)))

    def Sync(self) -> int:
        """Waits for the problem's stream and its side-stream label copies."""
        return lib().b40c_problem_sync(self._h)


class _Enactor:
    STRATEGY: Strategy

    def __init__(self, DEBUG: bool = False, INSTRUMENT: bool = False):
        h = ctypes.c_void_p()
        check(lib().b40c_enactor_create(int(self.STRATEGY), int(INSTRUMENT), int(DEBUG), ctypes.byref(h)))
        self._h = h
        self.DEBUG = DEBUG
        self.INSTRUMENT = INSTRUMENT

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().b40c_enactor_destroy(h)
            except Exception:
                pass
            self._h = None

    close = __del__

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def GetFrontierType(self) -> FrontierType:
        ft = ctypes.c_int()
        check(lib().b40c_enactor_frontier_type(self._h, ctypes.byref(ft)))
        return FrontierType(ft.value)

    def EnactSearch(self, problem: CsrProblem, src: int, max_grid_size: int = 0) -> int:
        return lib().b40c_enact_search(self._h, problem.handle, int(src), int(max_grid_size), Variant.DEFAULT)

    def EnactFusedSearch(self, problem: CsrProblem, src: int, max_grid_size: int = 0) -> int:
        return lib().b40c_enact_search(self._h, problem.handle, int(src), int(max_grid_size), Variant.FUSED)

    def EnactIterativeSearch(self, problem: CsrProblem, src: int, max_grid_size: int = 0) -> int:
        return lib().b40c_enact_search(self._h, problem.handle, int(src), int(max_grid_size), Variant.ITERATIVE)

    def EnactSearchAsync(self, problem: CsrProblem, src: int, max_grid_size: int = 0,
                         variant: int = Variant.DEFAULT) -> int:
        return lib().b40c_enact_search_async(self._h, problem.handle, int(src), int(max_grid_size), int(variant))

    def Sync(self) -> int:
        return lib().b40c_enactor_sync(self._h)

    def GetStatistics(self):
        """(total_queued, search_depth, avg_duty); search_depth = iteration - 1."""
        tq, sd, duty = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_double()
        check(lib().b40c_enactor_get_statistics(self._h, ctypes.byref(tq), ctypes.byref(sd), ctypes.byref(duty)))
        return tq.value, sd.value, duty.value

    def last_elapsed_ms(self) -> float:
        ms = ctypes.c_float()
        check(lib().b40c_enactor_last_elapsed_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def set_stream(self, stream_handle: int | None) -> None:
        check(lib().b40c_enactor_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    def set_policy(self, cta_threads: int = 0, warp_gather_threshold: int = 0, cta_gather_threshold: int = 0,
                   cull_flags: int = -1) -> None:
        """KernelPolicy knobs: CTA size, warp / CTA gather thresholds (edges; 0 keeps),
        cull flags (bit0 warp cull, bit1 history cache; -1 keeps)."""
        check(lib().b40c_enactor_set_policy(self._h, cta_threads, warp_gather_threshold, cta_gather_threshold,
                                            cull_flags))

    def set_level_log(self, enable: bool = True) -> None:
        check(lib().b40c_enactor_set_level_log(self._h, int(enable)))

    def level_log(self, max_records: int = 4096) -> list:
        """Per-level records of the last search: start time (ns, relative to the
        first level), input frontier queue length, input CTA and warp chunks,
        and whether the level ran bottom-up."""
        ts = (ctypes.c_int64 * max_records)()
        fr = (ctypes.c_int * max_records)()
        ch = (ctypes.c_int * max_records)()
        wc = (ctypes.c_int * max_records)()
        bu = (ctypes.c_int * max_records)()
        n = ctypes.c_int()
        check(lib().b40c_enactor_level_log(self._h, max_records, ts, fr, ch, wc, bu, ctypes.byref(n)))
        if n.value == 0:
            return []
        t0 = ts[0]
        we = (ctypes.c_int64 * max_records)()
        m = ctypes.c_int()
        check(lib().b40c_enactor_level_times(self._h, max_records, None, we, ctypes.byref(m)))
        return [{"level": i, "start_ns": ts[i] - t0, "frontier": fr[i], "chunks": ch[i], "wchunks": wc[i],
                 "bottom_up": bool(bu[i]), "work_end_ns": (we[i] - t0) if we[i] else None}
                for i in range(n.value)]

    def set_direction_optimizing(self, alpha: int = 14, beta: int = 24) -> None:
        """Bottom-up levels for fused expand-contract searches (alpha = 0: off)."""
        check(lib().b40c_enactor_set_direction_optimizing(self._h, int(alpha), int(beta)))

    def set_wait_limit_us(self, us: int) -> None:
        check(lib().b40c_enactor_set_wait_limit_us(self._h, int(us)))

    def set_bottom_up_staging(self, enable: bool = True) -> None:
        """Bottom-up steps stage their inputs in shared memory one step ahead (default off)."""
        check(lib().b40c_enactor_set_bottom_up_staging(self._h, int(bool(enable))))

    def set_narrow_levels(self, team_ctas: int, max_frontier: int, grid_frontier: int = 0) -> None:
        """Fused searches: the first levels of at most max_frontier queued
        entries run on one cluster of team_ctas CTAs (0: none), and
        (contract-expand, hybrid) full-grid levels of at most grid_frontier
        queued entries run the latency-first level body (0: none).  Both off
        by default."""
        check(lib().b40c_enactor_set_narrow_levels(self._h, int(team_ctas), int(max_frontier), int(grid_frontier)))

    def narrow_team(self) -> int:
        """CTAs of the cluster narrow levels run on (0: off or none fits)."""
        t = ctypes.c_int(0)
        check(lib().b40c_enactor_narrow_team(self._h, ctypes.byref(t)))
        return t.value

    def set_l2_persistence(self, what: int) -> None:
        """0 off, 1 keep the visited mask L2-resident, 2 the mask and the labels."""
        check(lib().b40c_enactor_set_l2_persistence(self._h, int(what)))


class EnactorExpandContract(_Enactor):
    """bfs::EnactorExpandContract<INSTRUMENT> (enactor_expand_contract.cuh:59-526)."""
    STRATEGY = Strategy.EXPAND_CONTRACT


class EnactorContractExpand(_Enactor):
    """bfs::EnactorContractExpand<INSTRUMENT> (enactor_contract_expand.cuh:61-598)."""
    STRATEGY = Strategy.CONTRACT_EXPAND


class EnactorTwoPhase(_Enactor):
    """bfs::EnactorTwoPhase<INSTRUMENT> (enactor_two_phase.cuh:68-766)."""
    STRATEGY = Strategy.TWO_PHASE


class EnactorHybrid(_Enactor):
    """bfs::EnactorHybrid<INSTRUMENT> (enactor_hybrid.cuh:64-758): contract-expand
    levels while the edge frontier is small, two-phase levels while it is large."""
    STRATEGY = Strategy.HYBRID


ENACTORS = {
    Strategy.EXPAND_CONTRACT: EnactorExpandContract,
    Strategy.CONTRACT_EXPAND: EnactorContractExpand,
    Strategy.TWO_PHASE: EnactorTwoPhase,
    Strategy.HYBRID: EnactorHybrid,
}


def make_enactor(strategy: int, **kw) -> _Enactor:
    return ENACTORS[Strategy(strategy)](**kw)


def debug_barrier_timeout(grid_size: int, wait_limit_us: int) -> int:
    """Runs the barrier-timeout probe; returns its cudaError_t (702 expected)."""
    return lib().b40c_debug_barrier_timeout(int(grid_size), int(wait_limit_us))


def version() -> str:
    v = lib().b40c_version()
    return v.decode() if v else ""
