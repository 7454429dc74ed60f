"""CPU tests of the oracle: pinned to the reference's own outputs (golden files,
and oracle/_ref when built), and able to catch planted mistakes."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_paths, load_golden


@pytest.mark.parametrize("path", golden_paths(), ids=lambda p: p.stem)
def test_oracle_matches_reference_golden(oracle, path):
    g, sources, labels, depths = load_golden(path)
    for i, s in enumerate(sources):
        lab, depth = oracle.bfs(g, int(s))
        assert np.array_equal(lab, labels[i])
        assert depth == depths[i]


def test_golden_set_is_complete():
    names = {p.stem for p in golden_paths()}
    assert {"ref_grid2d_32", "ref_grid3d_10", "ref_random_2000_u", "ref_random_3000_d",
            "ref_rmat_4096_u", "pkg_rmat_s12"} <= names


def _ref():
    from oracle import ReferenceBfs
    if not ReferenceBfs.available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    return ReferenceBfs()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_reference_binary(oracle, seed):
    """Restatement vs the reference's compiled SimpleReferenceBfs on fresh graphs."""
    ref = _ref()
    from back40computing_b200 import graphs
    row, col = ref.random(3000 + seed, 7000, seed % 2, seed)
    g = graphs.CsrGraph(row, col)
    for s in (0, 1, g.nodes - 1):
        a, da = oracle.bfs(g, s)
        b, db = ref.bfs(g, s)
        assert np.array_equal(a, b) and da == db


def test_visit_stats(oracle):
    from back40computing_b200 import graphs
    g = graphs.grid2d(10)
    lab, _ = oracle.bfs(g, 0)
    nv, ev = oracle.visit_stats(g, lab)
    assert nv == 100 and ev == g.edges


def _bfs_tree(g, src, depths):
    """A valid predecessor labelling built on the host from reference depths."""
    preds = np.full(g.nodes, -1, np.int32)
    preds[src] = -2
    for v in range(g.nodes):
        if depths[v] > 0:
            for e in range(g.row_offsets[v], g.row_offsets[v + 1]):
                u = g.column_indices[e]
                if depths[u] == depths[v] - 1:
                    preds[v] = u
                    break
    return preds


def test_predecessor_checker_catches_planted_mistakes(oracle):
    from back40computing_b200 import graphs
    g = graphs.grid2d(12)
    src = 0
    depths, _ = oracle.bfs(g, src)
    preds = _bfs_tree(g, src, depths)
    assert oracle.check_predecessors(g, preds, depths) == (-1, 0)
    far = int(np.argmax(depths))
    bad = preds.copy()
    bad[far] = -1                      # parentless node with positive depth
    assert oracle.check_predecessors(g, bad, depths) == (far, 1)
    bad = preds.copy()
    bad[far] = src                     # parent at the wrong depth
    assert oracle.check_predecessors(g, bad, depths)[1] == 2
    v = 13                             # depth 2 in a 12-wide grid: (1, 1)
    same_depth_nonneighbor = int(np.nonzero((depths == depths[v] - 1))[0][-1])
    bad = preds.copy()
    bad[v] = same_depth_nonneighbor    # right depth, but not adjacent
    if same_depth_nonneighbor not in g.column_indices[g.row_offsets[v]:g.row_offsets[v + 1]]:
        assert oracle.check_predecessors(g, bad, depths) == (v, 3)


def test_label_compare_finds_first_difference(oracle):
    a = np.arange(100, dtype=np.int32)
    b = a.copy()
    assert oracle.first_mismatch(a, b) == -1
    b[37] = -1
    b[80] = 5
    assert oracle.first_mismatch(a, b) == 37


def test_oracle_threads_agree(oracle):
    from back40computing_b200 import graphs
    g = graphs.rmat(11, 8, seed=4)
    src = g.sample_sources(9, 1)
    ev1 = oracle.bfs_many(g, src, 1)
    ev4 = oracle.bfs_many(g, src, 4)
    assert np.array_equal(ev1, ev4)
    for s, ev in zip(src, ev1):
        lab, _ = oracle.bfs(g, int(s))
        assert oracle.visit_stats(g, lab)[1] == ev


@pytest.mark.parametrize("scale,ef,undirected,seed", [(10, 16, True, 3), (12, 8, False, 5), (16, 16, True, 1)])
def test_oracle_rmat_matches_product_generator(scale, ef, undirected, seed):
    """The oracle's restated R-MAT (the CPU legs' input) is the product's graph,
    byte for byte, and draws the same sources."""
    import back40computing_b200 as b
    from oracle import rmat
    g_oracle = rmat(scale, ef, seed=seed, undirected=undirected)
    g_prod = b.rmat(scale, ef, 0.57, 0.19, 0.19, seed=seed, undirected=undirected)
    assert g_oracle.sha256() == g_prod.sha256()
    assert np.array_equal(g_oracle.sample_sources(64, 2), g_prod.sample_sources(64, 2))


def test_oracle_rmat_matches_product_generator_at_bench_size():
    """The bench workload itself: R-MAT scale 22, edge factor 16, seed 1,
    symmetrized (134,214,152 entries), and its 64 sources (seed 2)."""
    import back40computing_b200 as b
    from oracle import rmat
    g_oracle = rmat(22, 16, seed=1, undirected=True)
    g_prod = b.rmat(22, 16, 0.57, 0.19, 0.19, seed=1, undirected=True)
    assert g_oracle.edges == 134214152
    assert g_oracle.sha256() == g_prod.sha256()
    assert np.array_equal(g_oracle.sample_sources(64, 2), g_prod.sample_sources(64, 2))


def test_oracle_many_labels_match_single_searches(oracle):
    from oracle import rmat
    g = rmat(13, 8, seed=7)
    src = g.sample_sources(9, 3)
    labels, depths = oracle.bfs_many_labels(g, src, threads=4)
    for i, s in enumerate(src):
        lab, d = oracle.bfs(g, int(s))
        assert np.array_equal(labels[i], lab)
        assert depths[i] == d
