"""Serving with continuous batching: each query's result must be the same
alone and in the mix (bit-exact labels against the oracle), whatever runs
beside it and whenever it is admitted."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graphs():
    import back40computing_b200 as b
    return [b.rmat(12, 16, seed=1), b.grid2d(64), b.rmat(14, 8, seed=2), b.grid3d(16),
            b.erdos_renyi(4000, 16 / 3999, seed=3)]


def _trace(graphs, n, rate, seed):
    from back40computing_b200.serve import poisson_arrivals
    rng = np.random.default_rng(seed)
    gids = rng.integers(0, len(graphs), n).astype(np.int32)
    srcs = np.array([int(graphs[g].sample_sources(1, seed * 1000 + i)[0]) for i, g in enumerate(gids)], np.int32)
    return gids, srcs, poisson_arrivals(n, rate, seed)


def _server(graphs, **kw):
    from back40computing_b200.serve import BfsServer
    srv = BfsServer(**kw)
    for g in graphs:
        srv.add_graph(g)
    return srv


@pytest.mark.parametrize("rate", [2000.0, 200000.0])
def test_results_same_alone_and_in_the_mix(cuda_device, oracle, graphs, rate):
    srv = _server(graphs, max_slots=64, hbm_budget_bytes=256 << 20)
    gids, srcs, arr = _trace(graphs, 60, rate, seed=5)
    lat, span, labels = srv.run_trace(gids, srcs, arr, keep_labels=True)
    for i, (g, s) in enumerate(zip(gids, srcs)):
        alone, _ = oracle.bfs(graphs[g], int(s))
        assert oracle.first_mismatch(labels[i], alone) == -1, (i, g, s)
    assert (lat >= 0).all() and span >= arr[-1]
    st = srv.stats()
    assert st["epochs"] > 0
    if rate > 100000:
        assert st["max_active"] > 1  # queries overlapped on the device


def test_memory_bound_admission(cuda_device, oracle, graphs):
    """A budget that holds only a few searches at once still answers all, in order of capacity."""
    srv = _server(graphs, max_slots=256, hbm_budget_bytes=24 << 20)
    gids, srcs, arr = _trace(graphs, 40, 1e6, seed=9)
    lat, span, labels = srv.run_trace(gids, srcs, arr, keep_labels=True)
    for i, (g, s) in enumerate(zip(gids, srcs)):
        alone, _ = oracle.bfs(graphs[g], int(s))
        assert oracle.first_mismatch(labels[i], alone) == -1
    assert srv.stats()["max_active"] < 40


def test_one_slot_is_sequential(cuda_device, oracle, graphs):
    srv = _server(graphs, max_slots=1, hbm_budget_bytes=64 << 20)
    gids, srcs, arr = _trace(graphs, 8, 1e6, seed=3)
    lat, span, labels = srv.run_trace(gids, srcs, arr, keep_labels=True)
    for i, (g, s) in enumerate(zip(gids, srcs)):
        alone, _ = oracle.bfs(graphs[g], int(s))
        assert oracle.first_mismatch(labels[i], alone) == -1
    assert srv.stats()["max_active"] == 1
    assert np.all(np.diff(arr + lat) >= -1.0)  # FIFO completion


def test_epoch_length_does_not_change_results(cuda_device, oracle, graphs):
    for epoch in (1, 3, 1000):
        srv = _server(graphs, max_slots=32, hbm_budget_bytes=128 << 20)
        srv.set_policy(epoch_levels=epoch)
        gids, srcs, arr = _trace(graphs, 20, 50000.0, seed=epoch)
        _, _, labels = srv.run_trace(gids, srcs, arr, keep_labels=True)
        for i, (g, s) in enumerate(zip(gids, srcs)):
            alone, _ = oracle.bfs(graphs[g], int(s))
            assert oracle.first_mismatch(labels[i], alone) == -1


def test_trace_validation(cuda_device, graphs):
    from back40computing_b200.bfs import BfsError
    srv = _server(graphs[:1], max_slots=4, hbm_budget_bytes=16 << 20)
    with pytest.raises(BfsError):
        srv.run_trace([0, 0], [1, 2], [5.0, 1.0])
    with pytest.raises(BfsError):
        srv.run_trace([3], [1], [0.0])


@pytest.mark.parametrize("alpha,beta", [(0, 0), (1, 1)], ids=["top-down", "eager-bottom-up"])
def test_direction_switch_does_not_change_results(cuda_device, oracle, graphs, alpha, beta):
    srv = _server(graphs, max_slots=48, hbm_budget_bytes=128 << 20)
    srv.set_direction_optimizing(alpha, beta)
    gids, srcs, arr = _trace(graphs, 40, 100000.0, seed=13)
    _, _, labels = srv.run_trace(gids, srcs, arr, keep_labels=True)
    for i, (g, s) in enumerate(zip(gids, srcs)):
        alone, _ = oracle.bfs(graphs[g], int(s))
        assert oracle.first_mismatch(labels[i], alone) == -1
