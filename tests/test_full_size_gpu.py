"""Parity at the bench's full size: R-MAT scale 22, edge factor 16
(4,194,304 vertices, 134,214,152 entries), every strategy bit-exact against
the oracle, and properties that hold at any size (one label per reached
vertex, every edge spans at most one level, every reached vertex but the
source has a neighbour one level up)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def s22():
    import back40computing_b200 as b
    return b.rmat(22, 16, 0.57, 0.19, 0.19, seed=1, undirected=True)


def _level_properties(g, labels, src):
    row = g.row_offsets.astype(np.int64)
    col = g.column_indices
    u = np.repeat(np.arange(g.nodes), np.diff(row))
    lu, lv = labels[u], labels[col]
    reached = lu >= 0
    assert labels[src] == 0
    assert np.all(lv[reached] >= 0)                       # a reached vertex's neighbours are reached
    assert np.all(np.abs(lu[reached] - lv[reached]) <= 1)  # edges span at most one level
    has_parent = np.zeros(g.nodes, bool)
    up = reached & (lv == lu - 1)
    has_parent[u[up]] = True
    r = labels > 0
    assert np.all(has_parent[r])                           # every reached vertex has a parent one level up


def _check_sources(g, oracle, sources, strategies, chunk=16):
    """Every source, every strategy, bit-exact against the oracle's labels
    (computed over all host threads, `chunk` sources at a time)."""
    import back40computing_b200 as b
    prob = b.CsrProblem(False).from_graph(g)
    enactors = {s: b.make_enactor(s) for s in strategies}
    for c0 in range(0, len(sources), chunk):
        part = np.asarray(sources[c0:c0 + chunk], np.int32)
        refs, _ = oracle.bfs_many_labels(g, part)
        for i, s in enumerate(part):
            for strategy, en in enactors.items():
                b.check(prob.Reset(en.GetFrontierType(), 1.3))
                b.check(en.EnactSearch(prob, int(s)))
                labels = prob.labels()
                assert oracle.first_mismatch(labels, refs[i]) == -1, (strategy, int(s))
                if c0 == 0 and i == 0 and strategy == 0:
                    _level_properties(g, labels, int(s))
    prob.close()


def test_rmat22_headline_all_64_sources_bit_exact(cuda_device, oracle, s22):
    """The bench's headline: expand-contract (direction-optimizing) from all 64
    bench sources (seed 2), each bit-exact against the oracle."""
    _check_sources(s22, oracle, s22.sample_sources(64, 2), (0,))


def test_rmat22_other_strategies_8_sources_bit_exact(cuda_device, oracle, s22):
    """Contract-expand, two-phase and hybrid from the first 8 bench sources."""
    _check_sources(s22, oracle, s22.sample_sources(64, 2)[:8], (1, 2, 3))


def test_rmat22_predecessors_valid(cuda_device, oracle, s22):
    import back40computing_b200 as b
    g = s22
    s = int(g.sample_sources(1, 9)[0])
    ref, _ = oracle.bfs(g, s)
    prob = b.CsrProblem(True).from_graph(g)
    for strategy in (0, 1):
        en = b.make_enactor(strategy)
        b.check(prob.Reset(en.GetFrontierType(), 1.3))
        b.check(en.EnactSearch(prob, s))
        assert oracle.check_predecessors(g, prob.labels(), ref)[0] == -1, strategy


def test_grid3d_256_fused_and_per_level(cuda_device, oracle):
    """The high-diameter case: grid3d 256^3 from the corner (765 levels), every
    strategy in the persistent kernel and in per-level launches, bit-exact."""
    import back40computing_b200 as b
    g = b.grid3d(256)
    ref, _ = oracle.bfs(g, 0)
    assert int(ref.max()) == 765
    prob = b.CsrProblem(False).from_graph(g)
    for strategy in (0, 1, 2, 3):
        for variant in (1, 2):
            en = b.make_enactor(strategy)
            b.check(prob.Reset(en.GetFrontierType(), 1.3))
            b.check(en.EnactFusedSearch(prob, 0) if variant == 1 else en.EnactIterativeSearch(prob, 0))
            assert oracle.first_mismatch(prob.labels(), ref) == -1, (strategy, variant)
