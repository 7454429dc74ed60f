"""Host CSR graphs and their builders (the inputs of the BFS path).

``CsrGraph`` plays the role of b40c::graph::CsrGraph<int,int,int>
(b40c/graph/csr_graph.cuh:50-245).  The builders call the C++ generators of
libb40c_bfs (back40computing_b200/csrc/graph_gen.cpp); see that file for how
they relate to the reference builders in b40c/graph/builder/.
"""
from __future__ import annotations

import ctypes
import hashlib
from dataclasses import dataclass

import numpy as np

from ._lib import CsrT, last_error, lib


class GraphError(RuntimeError):
    pass


@dataclass
class CsrGraph:
    """int32 CSR: row_offsets[nodes + 1], column_indices[edges]."""
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

    def as_ctypes(self) -> CsrT:
        """A b40c_csr_t view of the arrays (valid while self is alive)."""
        c = CsrT()
        c.nodes = self.nodes
        c.edges = self.edges
        c.row_offsets = self.row_offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        c.column_indices = self.column_indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        return c

    def sample_sources(self, count: int, seed: int) -> np.ndarray:
        """count sources drawn with a seeded RNG among vertices of degree > 0."""
        out = np.empty(count, np.int32)
        c = self.as_ctypes()
        rc = lib().b40c_graph_sample_sources(ctypes.byref(c), count, seed, out.ctypes.data_as(ctypes.c_void_p))
        if rc:
            raise GraphError(last_error())
        return out


def _take(c: CsrT, name: str) -> CsrGraph:
    try:
        n, m = int(c.nodes), int(c.edges)
        row = np.ctypeslib.as_array(c.row_offsets, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(c.column_indices, shape=(m,)).copy() if m else np.zeros(0, np.int32)
    finally:
        lib().b40c_csr_free(ctypes.byref(c))
    return CsrGraph(row.astype(np.int32, copy=False), col.astype(np.int32, copy=False), name)


def _call(fn, *args, name: str) -> CsrGraph:
    c = CsrT()
    rc = fn(*args, ctypes.byref(c))
    if rc:
        raise GraphError(f"{name}: {last_error()} (code {rc})")
    return _take(c, name)


def grid2d(width: int, self_loops: bool = False) -> CsrGraph:
    """width x width 4-neighbour lattice, both directions stored."""
    return _call(lib().b40c_graph_grid2d, width, int(self_loops), name=f"grid2d-{width}")


def grid3d(width: int, self_loops: bool = False) -> CsrGraph:
    """width^3 6-neighbour lattice, both directions stored."""
    return _call(lib().b40c_graph_grid3d, width, int(self_loops), name=f"grid3d-{width}")


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1, undirected: bool = True) -> CsrGraph:
    """Graph500-style R-MAT, self-loops removed, duplicates kept, symmetrized."""
    return _call(lib().b40c_graph_rmat, scale, edge_factor, a, b, c, seed, int(undirected),
                 name=f"rmat-s{scale}-ef{edge_factor}-seed{seed}")


def erdos_renyi(nodes: int, p: float, seed: int = 1) -> CsrGraph:
    """Undirected G(n, p) without self-loops or parallel edges."""
    return _call(lib().b40c_graph_erdos_renyi, nodes, p, seed, name=f"er-n{nodes}-seed{seed}")


def from_coo(nodes: int, rows, cols) -> CsrGraph:
    """CSR from a COO edge list, stable by row (CsrGraph::FromCoo)."""
    r = np.ascontiguousarray(rows, dtype=np.int32)
    cc = np.ascontiguousarray(cols, dtype=np.int32)
    if r.shape != cc.shape:
        raise GraphError("rows and cols differ in length")
    return _call(lib().b40c_graph_from_coo, nodes, r.shape[0], r.ctypes.data_as(ctypes.c_void_p),
                 cc.ctypes.data_as(ctypes.c_void_p), name="coo")


def read_market(path, undirected: bool = False) -> CsrGraph:
    """Matrix Market coordinate file (entry "a b" is the edge b-1 -> a-1)."""
    return _call(lib().b40c_graph_read_market, str(path).encode(), int(undirected), name=f"market:{path}")


def read_metis(path) -> CsrGraph:
    """METIS adjacency file (1-based neighbour lists, both directions stored)."""
    return _call(lib().b40c_graph_read_metis, str(path).encode(), name=f"metis:{path}")


def read_dimacs(path, undirected: bool = False) -> CsrGraph:
    """DIMACS shortest-path arc file ("p" line, "a u v w" arcs)."""
    return _call(lib().b40c_graph_read_dimacs, str(path).encode(), int(undirected), name=f"dimacs:{path}")
