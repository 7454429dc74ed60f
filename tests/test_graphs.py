"""CPU tests of the CSR builders (the inputs of the BFS path)."""
from __future__ import annotations

import numpy as np
import pytest

from back40computing_b200 import graphs


def _valid_csr(g):
    assert g.row_offsets[0] == 0 and g.row_offsets[-1] == g.edges
    assert (np.diff(g.row_offsets) >= 0).all()
    if g.edges:
        assert g.column_indices.min() >= 0 and g.column_indices.max() < g.nodes


def _symmetric(g):
    rows = np.repeat(np.arange(g.nodes, dtype=np.int64), np.diff(g.row_offsets))
    fwd = np.sort(rows * g.nodes + g.column_indices)
    bwd = np.sort(g.column_indices.astype(np.int64) * g.nodes + rows)
    return np.array_equal(fwd, bwd)


def test_grid_sizes_match_configs():
    g = graphs.grid2d(1024)
    assert (g.nodes, g.edges) == (1048576, 4190208)
    _valid_csr(g)
    g3 = graphs.grid3d(64)
    assert g3.nodes == 64 ** 3 and g3.edges == 6 * 63 * 64 * 64
    _valid_csr(g3)
    assert _symmetric(graphs.grid3d(9)) and _symmetric(graphs.grid2d(13))


def test_rmat_properties():
    g = graphs.rmat(14, 16, seed=1)
    _valid_csr(g)
    assert g.nodes == 1 << 14
    assert g.edges % 2 == 0 and g.edges <= 2 * 16 * (1 << 14)
    rows = np.repeat(np.arange(g.nodes), np.diff(g.row_offsets))
    assert not (rows == g.column_indices).any()  # self-loops removed
    assert _symmetric(g)
    deg = g.degrees()
    assert deg.max() > 50 * deg[deg > 0].mean()  # skewed
    assert g.sha256() == graphs.rmat(14, 16, seed=1).sha256()  # deterministic
    assert g.sha256() != graphs.rmat(14, 16, seed=2).sha256()


def test_rmat_generation_order_within_rows():
    """Row u lists forward edges (u, v) in generation order, then reversed ones."""
    g = graphs.rmat(6, 4, seed=3, undirected=False)
    _valid_csr(g)
    gu = graphs.rmat(6, 4, seed=3, undirected=True)
    for u in range(g.nodes):
        fwd = g.column_indices[g.row_offsets[u]:g.row_offsets[u + 1]]
        both = gu.column_indices[gu.row_offsets[u]:gu.row_offsets[u + 1]]
        assert np.array_equal(both[:len(fwd)], fwd)


def test_erdos_renyi():
    n = 20000
    g = graphs.erdos_renyi(n, 16 / (n - 1), seed=5)
    _valid_csr(g)
    assert abs(g.edges / n - 16) < 0.5
    rows = np.repeat(np.arange(n, dtype=np.int64), g.degrees())
    keys = rows * n + g.column_indices
    assert np.unique(keys).shape[0] == keys.shape[0]  # no parallel edges
    assert not (rows == g.column_indices).any()
    assert _symmetric(g)


def test_from_coo_stable():
    g = graphs.from_coo(4, [2, 0, 2, 1, 0], [1, 3, 0, 2, 1])
    assert list(g.row_offsets) == [0, 2, 3, 5, 5]
    assert list(g.column_indices) == [3, 1, 2, 1, 0]
    with pytest.raises(graphs.GraphError):
        graphs.from_coo(3, [0, 5], [1, 1])


def test_sample_sources_have_degree():
    g = graphs.rmat(12, 8, seed=1)
    s = g.sample_sources(64, 2)
    assert (g.degrees()[s] > 0).all()
    assert np.array_equal(s, g.sample_sources(64, 2))


def test_builder_errors():
    with pytest.raises(graphs.GraphError):
        graphs.grid2d(0)
    with pytest.raises(graphs.GraphError):
        graphs.rmat(0)


def _ref():
    from oracle import ReferenceBfs
    if not ReferenceBfs.available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    return ReferenceBfs()


@pytest.mark.parametrize("w", [1, 2, 5, 31])
def test_lattices_equal_reference_builders_with_self_loops(w):
    ref = _ref()
    for mine, theirs in ((graphs.grid2d(w, True), ref.grid2d(w)), (graphs.grid3d(w, True), ref.grid3d(w))):
        assert np.array_equal(mine.row_offsets, theirs[0])
        assert np.array_equal(mine.column_indices, theirs[1])


def test_from_coo_equals_reference():
    ref = _ref()
    rng = np.random.default_rng(3)
    r, c = rng.integers(0, 500, 4000), rng.integers(0, 500, 4000)
    mine = graphs.from_coo(500, r, c)
    row, col = ref.from_coo(500, r, c)
    assert np.array_equal(mine.row_offsets, row) and np.array_equal(mine.column_indices, col)
