"""ctypes access to the BFS oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module, as the checker; the product path (back40computing_b200) never does.

* :class:`Oracle` wraps liboracle_bfs.so, the plain-C restatement in
  oracle/bfs_oracle.c of the reference's SimpleReferenceBfs
  (test/bfs/test_bfs.cu:503-578) and validators (:343-440).
* :class:`ReferenceBfs` wraps oracle/_ref/libref_bfs.so, the reference's own
  test/bfs/test_bfs.cu compiled from its sources (oracle/Makefile), when present.
* :func:`rmat` / :class:`OracleGraph` build the seeded R-MAT benchmark input
  from oracle/graph_gen_oracle.c, a restatement of the product's generator
  pinned to it by sha256 in tests/test_oracle.py, so that the CPU legs of the
  benchmark never load the product library.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_int64, c_uint, c_uint64, c_void_p
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle_bfs.so"
REF_SO = HERE / "_ref" / "libref_bfs.so"


def _p(a: np.ndarray) -> c_void_p:
    return a.ctypes.data_as(c_void_p)


def build_oracle() -> Path:
    """Builds liboracle_bfs.so with gcc when missing or stale."""
    srcs = (HERE / "bfs_oracle.c", HERE / "graph_gen_oracle.c")
    if not ORACLE_SO.exists() or any(ORACLE_SO.stat().st_mtime < s.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE), "liboracle_bfs.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return ORACLE_SO


class Oracle:
    def __init__(self):
        self.lib = ctypes.CDLL(str(build_oracle()))
        L = self.lib
        L.oracle_bfs.restype = c_int64
        L.oracle_bfs.argtypes = [c_int64, c_void_p, c_void_p, c_int, c_void_p]
        L.oracle_compare_labels.restype = c_int64
        L.oracle_compare_labels.argtypes = [c_int64, c_void_p, c_void_p]
        L.oracle_check_predecessors.restype = c_int64
        L.oracle_check_predecessors.argtypes = [c_int64, c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_int)]
        L.oracle_visit_stats.restype = None
        L.oracle_visit_stats.argtypes = [c_int64, c_void_p, c_void_p, POINTER(c_int64), POINTER(c_int64)]
        L.oracle_bfs_many.restype = c_int
        L.oracle_bfs_many.argtypes = [c_int64, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]
        L.oracle_bfs_many_labels.restype = c_int
        L.oracle_bfs_many_labels.argtypes = [c_int64, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p,
                                             c_void_p]

    def bfs(self, g, src: int):
        """(labels, search_depth) as SimpleReferenceBfs computes them."""
        labels = np.empty(g.nodes, np.int32)
        depth = self.lib.oracle_bfs(g.nodes, _p(g.row_offsets), _p(g.column_indices), int(src), _p(labels))
        if depth < 0:
            raise ValueError(f"oracle_bfs failed ({depth})")
        return labels, int(depth)

    def first_mismatch(self, computed: np.ndarray, reference: np.ndarray) -> int:
        return int(self.lib.oracle_compare_labels(reference.shape[0], _p(computed), _p(reference)))

    def check_predecessors(self, g, preds: np.ndarray, ref_depths: np.ndarray):
        """(-1, 0) when valid, else (first bad node, reason 1..3)."""
        reason = c_int()
        bad = self.lib.oracle_check_predecessors(g.nodes, _p(g.row_offsets), _p(g.column_indices), _p(preds),
                                                 _p(ref_depths), ctypes.byref(reason))
        return int(bad), reason.value

    def visit_stats(self, g, labels: np.ndarray):
        """(nodes_visited, edges_visited) as DisplayStats counts them."""
        nv, ev = c_int64(), c_int64()
        self.lib.oracle_visit_stats(g.nodes, _p(g.row_offsets), _p(labels), ctypes.byref(nv), ctypes.byref(ev))
        return nv.value, ev.value

    def bfs_many(self, g, sources: np.ndarray, threads: int) -> np.ndarray:
        """Independent searches over host threads; returns edges_visited per source."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        ev = np.zeros(src.shape[0], np.int64)
        rc = self.lib.oracle_bfs_many(g.nodes, _p(g.row_offsets), _p(g.column_indices), _p(src), src.shape[0],
                                      int(threads), _p(ev))
        if rc:
            raise MemoryError("oracle_bfs_many")
        return ev


    def bfs_many_labels(self, g, sources, threads: int = 0):
        """(labels[len(sources), nodes], search_depths) of SimpleReferenceBfs
        from every source, computed on `threads` host threads (0 = all)."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        labels = np.empty((src.shape[0], g.nodes), np.int32)
        depths = np.zeros(src.shape[0], np.int64)
        threads = threads or os.cpu_count() or 1
        self.lib.oracle_bfs_many_labels(g.nodes, _p(g.row_offsets), _p(g.column_indices), _p(src), src.shape[0],
                                        int(threads), _p(labels), _p(depths))
        if np.any(depths < 0):
            raise ValueError("oracle_bfs_many_labels: bad source")
        return labels, depths


@dataclass
class OracleGraph:
    """int32 CSR built by the oracle's restated generators."""
    row_offsets: np.ndarray
    column_indices: np.ndarray
    name: str = ""

    @property
    def nodes(self) -> int:
        return int(self.row_offsets.shape[0] - 1)

    @property
    def edges(self) -> int:
        return int(self.column_indices.shape[0])

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_offsets)

    def sha256(self) -> str:
        h = hashlib.sha256()
        h.update(np.ascontiguousarray(self.row_offsets).tobytes())
        h.update(np.ascontiguousarray(self.column_indices).tobytes())
        return h.hexdigest()

    def sample_sources(self, count: int, seed: int) -> np.ndarray:
        out = np.empty(count, np.int32)
        lib = Oracle().lib
        lib.oracle_sample_sources.restype = c_int
        lib.oracle_sample_sources.argtypes = [c_int64, c_void_p, c_int, c_uint64, c_void_p]
        if lib.oracle_sample_sources(self.nodes, _p(self.row_offsets), int(count), int(seed), _p(out)):
            raise ValueError("oracle_sample_sources: graph has no edges")
        return out


def rmat(scale: int, edge_factor: int, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1,
         undirected: bool = True, threads: int = 0) -> OracleGraph:
    """The seeded R-MAT benchmark graph (oracle/graph_gen_oracle.c)."""
    lib = Oracle().lib
    lib.oracle_rmat.restype = c_int
    lib.oracle_rmat.argtypes = [c_int, c_int, c_double, c_double, c_double, c_uint64, c_int, c_int,
                                POINTER(c_int64), POINTER(c_int64), POINTER(POINTER(c_int)), POINTER(POINTER(c_int))]
    lib.oracle_free.argtypes = [c_void_p]
    lib.oracle_free.restype = None
    n, m = c_int64(), c_int64()
    ro, ci = POINTER(c_int)(), POINTER(c_int)()
    if lib.oracle_rmat(scale, edge_factor, a, b, c, seed, int(undirected), int(threads or os.cpu_count() or 1),
                       ctypes.byref(n), ctypes.byref(m), ctypes.byref(ro), ctypes.byref(ci)):
        raise ValueError("oracle_rmat: invalid arguments or allocation failure")
    try:
        row = np.ctypeslib.as_array(ro, (n.value + 1,)).copy()
        col = np.ctypeslib.as_array(ci, (m.value,)).copy() if m.value else np.zeros(0, np.int32)
    finally:
        lib.oracle_free(ctypes.cast(ro, c_void_p))
        lib.oracle_free(ctypes.cast(ci, c_void_p))
    return OracleGraph(row, col, f"rmat-s{scale}-ef{edge_factor}")


class ReferenceBfs:
    """The reference's own CPU BFS and builders (oracle/_ref), when built."""

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def __init__(self):
        self.lib = ctypes.CDLL(str(REF_SO))
        L = self.lib
        L.ref_simple_bfs.restype = c_int
        L.ref_simple_bfs.argtypes = [c_int, c_int, c_void_p, c_void_p, c_int, c_void_p]
        L.ref_simple_bfs_many.restype = c_int
        L.ref_simple_bfs_many.argtypes = [c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]
        gp = [POINTER(c_int64), POINTER(c_int64), POINTER(POINTER(c_int)), POINTER(POINTER(c_int))]
        L.ref_build_grid2d.argtypes = [c_int] + gp
        L.ref_build_grid3d.argtypes = [c_int] + gp
        L.ref_build_random.argtypes = [c_int, c_int, c_int, c_uint] + gp
        L.ref_build_rmat.argtypes = [c_int, c_int, c_int, c_double, c_double, c_double, c_uint] + gp
        L.ref_from_coo.argtypes = [c_int, c_int, c_void_p, c_void_p] + gp
        L.ref_read_market.argtypes = [ctypes.c_char_p, c_int] + gp
        L.ref_read_metis.argtypes = [ctypes.c_char_p] + gp
        L.ref_read_dimacs.argtypes = [ctypes.c_char_p, c_int] + gp
        L.ref_free.argtypes = [c_void_p]
        L.ref_free.restype = None

    def bfs(self, g, src: int):
        labels = np.empty(g.nodes, np.int32)
        depth = self.lib.ref_simple_bfs(g.nodes, g.edges, _p(g.row_offsets), _p(g.column_indices), int(src),
                                        _p(labels))
        return labels, int(depth)

    def bfs_many(self, g, sources: np.ndarray, threads: int) -> np.ndarray:
        src = np.ascontiguousarray(sources, dtype=np.int32)
        ev = np.zeros(src.shape[0], np.int64)
        self.lib.ref_simple_bfs_many(g.nodes, g.edges, _p(g.row_offsets), _p(g.column_indices), _p(src),
                                     src.shape[0], int(threads), _p(ev))
        return ev

    def _graph(self, fn, *args):
        n, m = c_int64(), c_int64()
        ro, ci = POINTER(c_int)(), POINTER(c_int)()
        rc = fn(*args, ctypes.byref(n), ctypes.byref(m), ctypes.byref(ro), ctypes.byref(ci))
        if rc:
            raise RuntimeError("reference builder failed")
        try:
            row = np.ctypeslib.as_array(ro, (n.value + 1,)).copy()
            col = np.ctypeslib.as_array(ci, (m.value,)).copy() if m.value else np.zeros(0, np.int32)
        finally:
            self.lib.ref_free(ctypes.cast(ro, c_void_p))
            self.lib.ref_free(ctypes.cast(ci, c_void_p))
        return row.astype(np.int32), col.astype(np.int32)

    def grid2d(self, width):
        return self._graph(self.lib.ref_build_grid2d, width)

    def grid3d(self, width):
        return self._graph(self.lib.ref_build_grid3d, width)

    def random(self, nodes, edges, undirected, seed):
        return self._graph(self.lib.ref_build_random, nodes, edges, int(undirected), seed)

    def rmat(self, nodes, edges, undirected, a, b, c, seed):
        return self._graph(self.lib.ref_build_rmat, nodes, edges, int(undirected), a, b, c, seed)

    def from_coo(self, nodes, rows, cols):
        r = np.ascontiguousarray(rows, dtype=np.int32)
        cc = np.ascontiguousarray(cols, dtype=np.int32)
        return self._graph(self.lib.ref_from_coo, nodes, r.shape[0], _p(r), _p(cc))

    def read_market(self, path, undirected):
        return self._graph(self.lib.ref_read_market, str(path).encode(), int(undirected))

    def read_metis(self, path):
        return self._graph(self.lib.ref_read_metis, str(path).encode())

    def read_dimacs(self, path, undirected):
        return self._graph(self.lib.ref_read_dimacs, str(path).encode(), int(undirected))
