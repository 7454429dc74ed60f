"""Batched multi-search BFS: every search of a batch must equal its own
single search (bit-exact depth labels against the oracle)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed_graphs():
    import back40computing_b200 as b
    return [b.rmat(10, 8, seed=1), b.rmat(13, 16, seed=2), b.erdos_renyi(3000, 16 / 2999, seed=3),
            b.grid2d(40), b.rmat(14, 24, seed=4), b.grid3d(12)]


def _check(oracle, batch, graphs, gids, srcs, mark_pred=False):
    for i, (g, s) in enumerate(zip(gids, srcs)):
        ref, _ = oracle.bfs(graphs[g], int(s))
        got = batch.labels(i)
        if mark_pred:
            assert oracle.check_predecessors(graphs[g], got, ref)[0] == -1, i
        else:
            assert oracle.first_mismatch(got, ref) == -1, (i, g, s)
            assert batch.search_depth(i) == int(ref.max())


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_matches_oracle(cuda_device, oracle, mixed_graphs, use_graph):
    from back40computing_b200.batch import BfsBatch
    batch = BfsBatch()
    ids = [batch.add_graph(g) for g in mixed_graphs]
    gids, srcs = [], []
    for gid, g in zip(ids, mixed_graphs):
        for s in g.sample_sources(5, 7 + gid):
            gids.append(gid)
            srcs.append(int(s))
    batch.run(gids, srcs, use_cuda_graph=use_graph)
    _check(oracle, batch, mixed_graphs, gids, srcs)
    # replay the same batch, then a different one
    batch.run(gids, srcs, use_cuda_graph=use_graph)
    _check(oracle, batch, mixed_graphs, gids, srcs)
    gids2, srcs2 = gids[::-1], [int(mixed_graphs[g].sample_sources(1, 99 + i)[0]) for i, g in enumerate(gids[::-1])]
    batch.run(gids2, srcs2, use_cuda_graph=use_graph)
    _check(oracle, batch, mixed_graphs, gids2, srcs2)


def test_batch_predecessors_valid(cuda_device, oracle, mixed_graphs):
    from back40computing_b200.batch import BfsBatch
    batch = BfsBatch(mark_predecessors=True)
    ids = [batch.add_graph(g) for g in mixed_graphs]
    gids = ids * 3
    srcs = [int(mixed_graphs[g].sample_sources(1, 5 + k)[0]) for k, g in enumerate(gids)]
    batch.run(gids, srcs)
    _check(oracle, batch, mixed_graphs, gids, srcs, mark_pred=True)


@pytest.mark.parametrize("policy", [dict(cta_threads=128), dict(cta_threads=256), dict(cta_threads=512),
                                    dict(warp_gather_threshold=8, cta_gather_threshold=64),
                                    dict(warp_gather_threshold=100000, cta_gather_threshold=100000),
                                    dict(cull_flags=0), dict(cull_flags=3)],
                         ids=lambda p: ",".join(f"{k}={v}" for k, v in p.items()))
def test_batch_policies(cuda_device, oracle, mixed_graphs, policy):
    from back40computing_b200.batch import BfsBatch
    batch = BfsBatch()
    batch.set_policy(**policy)
    ids = [batch.add_graph(g) for g in mixed_graphs]
    gids = ids * 2
    srcs = [int(mixed_graphs[g].sample_sources(1, 11 + k)[0]) for k, g in enumerate(gids)]
    batch.run(gids, srcs)
    _check(oracle, batch, mixed_graphs, gids, srcs)


def test_batch_edge_cases(cuda_device, oracle):
    import back40computing_b200 as b
    from back40computing_b200.batch import BfsBatch
    graphs = [b.from_coo(1, [], []), b.from_coo(5, [1, 2], [2, 1]),
              b.from_coo(20001, [0] * 20000 + list(range(1, 20001)), list(range(1, 20001)) + [0] * 20000)]
    batch = BfsBatch()
    ids = [batch.add_graph(g) for g in graphs]
    gids = [ids[0], ids[1], ids[1], ids[2], ids[2]]
    srcs = [0, 0, 1, 0, 777]
    batch.run(gids, srcs)
    _check(oracle, batch, graphs, gids, srcs)


@pytest.mark.parametrize("alpha,beta", [(0, 0), (1, 1), (14, 24), (1000, 1)],
                         ids=["top-down", "eager-bottom-up", "default", "late-bottom-up"])
def test_batch_direction_optimizing(cuda_device, oracle, mixed_graphs, alpha, beta):
    """Each search switches direction by its own frontier; a directed graph
    (which fails the symmetry check) stays top-down in the same batch."""
    from conftest import golden_paths, load_golden
    from back40computing_b200.batch import BfsBatch
    directed, _, _, _ = load_golden([p for p in golden_paths() if p.stem == "ref_random_3000_d"][0])
    graphs = list(mixed_graphs) + [directed]
    batch = BfsBatch()
    batch.set_direction_optimizing(alpha, beta)
    ids = [batch.add_graph(g) for g in graphs]
    gids = ids * 4
    srcs = [int(graphs[g].sample_sources(1, 31 + k)[0]) for k, g in enumerate(gids)]
    batch.run(gids, srcs, use_cuda_graph=True)
    _check(oracle, batch, graphs, gids, srcs)
    batch.run(gids, srcs, use_cuda_graph=True)  # replay
    _check(oracle, batch, graphs, gids, srcs)


def test_bench_batched_set_every_search_matches_oracle(cuda_device, oracle):
    """The bench's batched workload itself: 64 graphs (48 R-MAT of scale 12..20
    and edge factor 8..32, 16 Erdos-Renyi of mean degree 16), 16 seeded sources
    each, 1024 searches in one CUDA-graph launch with the tuned policy; every
    search's labels bit-exact against the oracle."""
    import bench
    from back40computing_b200 import tune
    from back40computing_b200.batch import BfsBatch
    gs, _, gids, srcs = bench.batched_set(max_scale=20)
    policy = tune.tune_batch(gs, gids, srcs, cache=tune.TuneCache(None, seed=tune.SHIPPED))
    batch = BfsBatch()
    tune.apply_batch_policy(batch, policy)
    for g in gs:
        batch.add_graph(g)
    batch.run(gids, srcs, use_cuda_graph=True)
    batch.run(gids, srcs, use_cuda_graph=True)  # the replayed graph, as the bench times it
    for gi, g in enumerate(gs):
        idx = np.nonzero(gids == gi)[0]
        refs, _ = oracle.bfs_many_labels(g, srcs[idx])
        for k, i in enumerate(idx):
            assert oracle.first_mismatch(batch.labels(int(i)), refs[k]) == -1, (gi, int(i), int(srcs[i]))
            assert batch.search_depth(int(i)) == int(refs[k].max())
    batch.close()


def test_replica_share_through_a_batch(cuda_device, oracle, mixed_graphs):
    """One replica's share (here, every query: one process) run by
    replicas.batch_share on a BfsBatch holding every graph, gathered in query
    order; each label array against the oracle."""
    from back40computing_b200.batch import BfsBatch
    from back40computing_b200.replicas import batch_share, run_partitioned
    batch = BfsBatch()
    for g in mixed_graphs:
        batch.add_graph(g)
    gids, srcs = [], []
    for gi, g in enumerate(mixed_graphs):
        for s in g.sample_sources(3, 71 + gi):
            gids.append(gi)
            srcs.append(int(s))
    costs = [mixed_graphs[g].edges for g in gids]
    labels, secs = run_partitioned(gids, srcs, batch_share(batch), costs=costs)
    assert len(secs) == 1 and secs[0] > 0
    for i, (g, s) in enumerate(zip(gids, srcs)):
        ref, _ = oracle.bfs(mixed_graphs[g], s)
        assert oracle.first_mismatch(labels[i], ref) == -1, i
    batch.close()
