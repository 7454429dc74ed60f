"""Serving BFS queries with continuous batching over resident graphs.

    server = BfsServer(max_slots=512, hbm_budget_bytes=16 << 30)
    gid = server.add_graph(g)
    lat_us, makespan_us = server.run_trace(graph_ids, sources, arrival_us)

The request loop runs in C++ inside libb40c_bfs (b40c_server_run_trace): it
admits arrived queries into free search slots while the HBM budget allows,
runs the admitted searches together in epochs of the multi-search kernel and
retires them as they finish.  poisson_arrivals() builds the arrival times of
a Poisson stream.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib
from .bfs import check
from .graphs import CsrGraph


def poisson_arrivals(n: int, rate_per_s: float, seed: int) -> np.ndarray:
    """Arrival times (µs) of n queries of a Poisson stream of the given rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1e6 / rate_per_s, n))


class BfsServer:
    def __init__(self, max_slots: int = 512, hbm_budget_bytes: int = 8 << 30, mark_predecessors: bool = False):
        h = ctypes.c_void_p()
        check(lib().b40c_server_create(int(mark_predecessors), int(max_slots), int(hbm_budget_bytes),
                                       ctypes.byref(h)))
        self._h = h
        self.graph_nodes: list[int] = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().b40c_server_destroy(h)
            except Exception:
                pass
            self._h = None

    close = __del__

    def add_graph(self, g: CsrGraph) -> int:
        gid = ctypes.c_int()
        check(lib().b40c_server_add_graph(self._h, g.nodes, g.edges, g.column_indices.ctypes.data_as(ctypes.c_void_p),
                                          g.row_offsets.ctypes.data_as(ctypes.c_void_p), ctypes.byref(gid)))
        self.graph_nodes.append(g.nodes)
        return gid.value

    def set_policy(self, cta_threads: int = 0, warp_gather_threshold: int = 0, cta_gather_threshold: int = 0,
                   cull_flags: int = -1, epoch_levels: int = 0) -> None:
        check(lib().b40c_server_set_policy(self._h, cta_threads, warp_gather_threshold, cta_gather_threshold,
                                           cull_flags, epoch_levels))

    def set_direction_optimizing(self, alpha: int = 14, beta: int = 24) -> None:
        """Bottom-up levels per query on symmetric graphs (alpha = 0: off)."""
        check(lib().b40c_server_set_direction_optimizing(self._h, int(alpha), int(beta)))

    def run_trace(self, graph_ids, sources, arrival_us, keep_labels: bool = False):
        """Replays the trace in real time; returns (latency_us, makespan_us[, labels])."""
        gids = np.ascontiguousarray(graph_ids, dtype=np.int32)
        srcs = np.ascontiguousarray(sources, dtype=np.int32)
        arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
        n = gids.shape[0]
        lat = np.zeros(n, np.float64)
        span = ctypes.c_double()
        outs = None
        ptrs = None
        if keep_labels:
            outs = [np.empty(self.graph_nodes[g], np.int32) for g in gids]
            ptrs = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
        check(lib().b40c_server_run_trace(self._h, n, gids.ctypes.data_as(ctypes.c_void_p),
                                          srcs.ctypes.data_as(ctypes.c_void_p), arr.ctypes.data_as(ctypes.c_void_p),
                                          lat.ctypes.data_as(ctypes.c_void_p), ptrs, ctypes.byref(span)))
        if keep_labels:
            return lat, span.value, outs
        return lat, span.value

    def stats(self):
        e, m = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().b40c_server_stats(self._h, ctypes.byref(e), ctypes.byref(m)))
        return {"epochs": e.value, "max_active": m.value}
