"""Batched BFS: many (graph, source) searches in one persistent launch.

The reference has no batched API (one search per EnactSearch); this is the
B200 build's multi-search path over the C ABI's b40c_batch_* calls:

    batch = BfsBatch()
    gid = batch.add_graph(g)                  # graphs stay resident
    batch.run([gid, gid, ...], [src0, src1, ...], use_cuda_graph=True)
    labels_i = batch.labels(i)                # int32 depth labels of search i
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib
from .bfs import check
from .graphs import CsrGraph


class BfsBatch:
    def __init__(self, mark_predecessors: bool = False):
        h = ctypes.c_void_p()
        check(lib().b40c_batch_create(int(mark_predecessors), ctypes.byref(h)))
        self._h = h
        self.graph_nodes: list[int] = []
        self._last = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().b40c_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    close = __del__

    def add_graph(self, g: CsrGraph) -> int:
        gid = ctypes.c_int()
        check(lib().b40c_batch_add_graph(self._h, g.nodes, g.edges, g.column_indices.ctypes.data_as(ctypes.c_void_p),
                                         g.row_offsets.ctypes.data_as(ctypes.c_void_p), ctypes.byref(gid)))
        self.graph_nodes.append(g.nodes)
        return gid.value

    def set_policy(self, cta_threads: int = 0, warp_gather_threshold: int = 0, cta_gather_threshold: int = 0,
                   cull_flags: int = -1) -> None:
        check(lib().b40c_batch_set_policy(self._h, cta_threads, warp_gather_threshold, cta_gather_threshold,
                                          cull_flags))

    def set_direction_optimizing(self, alpha: int = 14, beta: int = 24) -> None:
        """Bottom-up levels per search on symmetric graphs (alpha = 0: off)."""
        check(lib().b40c_batch_set_direction_optimizing(self._h, int(alpha), int(beta)))

    def set_stream(self, stream_handle: int | None) -> None:
        check(lib().b40c_batch_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    def _args(self, graph_ids, sources):
        gids = np.ascontiguousarray(graph_ids, dtype=np.int32)
        srcs = np.ascontiguousarray(sources, dtype=np.int32)
        if gids.shape != srcs.shape:
            raise ValueError("graph_ids and sources differ in length")
        self._last = (gids, srcs)
        return gids, srcs

    def run(self, graph_ids, sources, use_cuda_graph: bool = True) -> None:
        gids, srcs = self._args(graph_ids, sources)
        check(lib().b40c_batch_run(self._h, gids.shape[0], gids.ctypes.data_as(ctypes.c_void_p),
                                   srcs.ctypes.data_as(ctypes.c_void_p), int(use_cuda_graph)))

    def run_async(self, graph_ids, sources, use_cuda_graph: bool = True) -> None:
        gids, srcs = self._args(graph_ids, sources)
        check(lib().b40c_batch_run_async(self._h, gids.shape[0], gids.ctypes.data_as(ctypes.c_void_p),
                                         srcs.ctypes.data_as(ctypes.c_void_p), int(use_cuda_graph)))

    def sync(self) -> None:
        check(lib().b40c_batch_sync(self._h))

    def labels(self, search: int) -> np.ndarray:
        gid = int(self._last[0][search])
        out = np.empty(self.graph_nodes[gid], np.int32)
        check(lib().b40c_batch_extract(self._h, search, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def search_depth(self, search: int) -> int:
        d = ctypes.c_int()
        check(lib().b40c_batch_search_depth(self._h, search, ctypes.byref(d)))
        return d.value

    def last_elapsed_ms(self) -> float:
        ms = ctypes.c_float()
        check(lib().b40c_batch_last_elapsed_ms(self._h, ctypes.byref(ms)))
        return ms.value
