"""CPU tests of the graph-file readers, pinned to the reference's own readers
(BuildMarketGraph / BuildMetisGraph / BuildDimacsGraph via oracle/_ref)."""
from __future__ import annotations

import numpy as np
import pytest

from back40computing_b200 import graphs


def _edges(seed, n=300, m=1500):
    rng = np.random.default_rng(seed)
    return n, rng.integers(1, n + 1, m), rng.integers(1, n + 1, m)


def write_market(path, n, a, b):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n% comment\n")
        f.write(f"{n} {n} {len(a)}\n")
        for x, y in zip(a, b):
            f.write(f"{x} {y} 1\n")


def write_dimacs(path, n, a, b):
    with open(path, "w") as f:
        f.write("c generated\n")
        f.write(f"p sp {n} {len(a)}\n")
        for x, y in zip(a, b):
            f.write(f"a {x} {y} 7\n")


def write_metis(path, g):
    with open(path, "w") as f:
        f.write("% adjacency\n")
        f.write(f"{g.nodes} {g.edges // 2}\n")
        for v in range(g.nodes):
            nb = g.column_indices[g.row_offsets[v]:g.row_offsets[v + 1]] + 1
            f.write(" ".join(str(x) for x in nb) + "\n")


@pytest.mark.parametrize("undirected", [False, True])
def test_market_meaning(tmp_path, undirected):
    n, a, b = _edges(1)
    p = tmp_path / "g.mtx"
    write_market(p, n, a, b)
    g = graphs.read_market(p, undirected)
    rows, cols = [], []
    for x, y in zip(a, b):  # entry "x y" is the edge y-1 -> x-1, then its reverse
        rows.append(y - 1)
        cols.append(x - 1)
        if undirected:
            rows.append(x - 1)
            cols.append(y - 1)
    ref = graphs.from_coo(n, rows, cols)
    assert np.array_equal(g.row_offsets, ref.row_offsets) and np.array_equal(g.column_indices, ref.column_indices)


def test_readers_reject_bad_files(tmp_path):
    p = tmp_path / "bad.mtx"
    p.write_text("3 4 1\n1 2\n")
    with pytest.raises(graphs.GraphError, match="not square"):
        graphs.read_market(p)
    p.write_text("3 3 2\n1 2\n")
    with pytest.raises(graphs.GraphError, match="only 1 of 2"):
        graphs.read_market(p)
    q = tmp_path / "bad.gr"
    q.write_text("p sp 3 1\na 1 9 1\n")
    with pytest.raises(graphs.GraphError, match="bad arc"):
        graphs.read_dimacs(q)
    with pytest.raises(graphs.GraphError, match="cannot open"):
        graphs.read_metis(tmp_path / "missing.graph")


def _ref():
    from oracle import ReferenceBfs
    if not ReferenceBfs.available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    return ReferenceBfs()


@pytest.mark.parametrize("undirected", [False, True])
def test_market_equals_reference_reader(tmp_path, undirected):
    ref = _ref()
    n, a, b = _edges(2)
    # The reference keeps a directed file's order without sorting; give it rows in order.
    order = np.argsort(b, kind="stable")
    a, b = a[order], b[order]
    p = tmp_path / "g.mtx"
    write_market(p, n, a, b)
    mine = graphs.read_market(p, undirected)
    row, col = ref.read_market(p, undirected)
    assert np.array_equal(mine.row_offsets, row) and np.array_equal(mine.column_indices, col)


@pytest.mark.parametrize("undirected", [False, True])
def test_dimacs_equals_reference_reader(tmp_path, undirected):
    ref = _ref()
    n, a, b = _edges(3)
    order = np.argsort(a, kind="stable")
    a, b = a[order], b[order]
    p = tmp_path / "g.gr"
    write_dimacs(p, n, a, b)
    mine = graphs.read_dimacs(p, undirected)
    row, col = ref.read_dimacs(p, undirected)
    assert np.array_equal(mine.row_offsets, row) and np.array_equal(mine.column_indices, col)


def test_metis_equals_reference_reader(tmp_path):
    ref = _ref()
    g = graphs.erdos_renyi(400, 0.02, seed=4)
    p = tmp_path / "g.graph"
    write_metis(p, g)
    mine = graphs.read_metis(p)
    row, col = ref.read_metis(p)
    assert np.array_equal(mine.row_offsets, row) and np.array_equal(mine.column_indices, col)
    assert np.array_equal(mine.row_offsets, g.row_offsets) and np.array_equal(mine.column_indices, g.column_indices)
