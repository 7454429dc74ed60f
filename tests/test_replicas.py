"""Replica placement of batched and served queries (back40computing_b200.replicas)
on CPU: the partition itself, and two gloo ranks that each really search their
share of the queries (with the CPU oracle standing in for a rank's GPU) and
gather the results on rank 0, which checks every label array."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _graphs():
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import rmat
    return [rmat(9, 8, seed=1), rmat(11, 16, seed=2), rmat(10, 4, seed=3, undirected=False)]


def _queries(graphs):
    gids, srcs = [], []
    for gi, g in enumerate(graphs):
        for s in g.sample_sources(7, 50 + gi):
            gids.append(gi)
            srcs.append(int(s))
    return np.array(gids, np.int32), np.array(srcs, np.int32)


def test_partition_covers_every_query_once():
    from back40computing_b200.replicas import partition
    gids = np.arange(23) % 5
    costs = np.array([1, 50, 3, 7, 20])[gids]
    for world in (1, 2, 3, 8):
        for mode in ("round_robin", "load"):
            parts = partition(gids, world, costs, mode)
            assert len(parts) == world
            allq = np.sort(np.concatenate(parts))
            assert np.array_equal(allq, np.arange(23))
            assert all(np.all(np.diff(p) > 0) for p in parts)  # each share in query order
        loads = [costs[p].sum() for p in partition(gids, world, costs, "load")]
        # longest-first greedy: no rank exceeds the mean by more than the largest query
        assert max(loads) <= costs.sum() / world + costs.max()
    with pytest.raises(ValueError):
        partition(gids, 2, costs[:3])
    with pytest.raises(ValueError):
        partition(gids, 2, mode="random")


def test_single_process_runs_everything():
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle
    from back40computing_b200.replicas import run_partitioned, wall_share
    graphs = _graphs()
    gids, srcs = _queries(graphs)
    orc = Oracle()
    labels, secs = run_partitioned(gids, srcs, wall_share(lambda g, s: orc.bfs(graphs[g], s)[0]))
    assert len(secs) == 1
    for i, (g, s) in enumerate(zip(gids, srcs)):
        assert np.array_equal(labels[i], orc.bfs(graphs[g], int(s))[0])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _FakeServer:
    """A rank's request loop stand-in: serves its share one query at a time,
    each taking (source % 7 + 1) * 10 µs, FIFO from its arrival."""

    def run_trace(self, gids, srcs, arr):
        t, lat = 0.0, []
        for s, a in zip(srcs, arr):
            t = max(t, a) + (int(s) % 7 + 1) * 10.0
            lat.append(t - a)
        return np.array(lat), t


def _rank_main(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    from oracle import Oracle
    from back40computing_b200.replicas import run_partitioned, serve_partitioned, wall_share
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    graphs = _graphs()
    gids, srcs = _queries(graphs)
    costs = np.array([graphs[g].edges for g in gids], np.float64)
    orc = Oracle()
    ran = []

    def search(g, s):
        ran.append((g, s))
        return orc.bfs(graphs[g], s)[0]

    labels, secs = run_partitioned(gids, srcs, wall_share(search), costs=costs)
    arrivals = np.arange(len(gids), dtype=np.float64) * 5.0
    served = serve_partitioned(_FakeServer(), gids, srcs, arrivals)
    out[rank] = {"ran": ran, "labels": labels, "secs": secs, "served": served}
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_search_their_shares_and_gather():
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
        codes = [p.exitcode for p in procs]
        res = dict(out)
    assert codes == [0, 0], codes
    graphs = _graphs()
    gids, srcs = _queries(graphs)
    ran0, ran1 = set(res[0]["ran"]), set(res[1]["ran"])
    assert ran0 and ran1 and not (ran0 & ran1)                       # disjoint, non-empty shares
    assert ran0 | ran1 == {(int(g), int(s)) for g, s in zip(gids, srcs)}
    assert res[1]["labels"] is None and res[1]["served"] is None     # gathered on rank 0 only
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle
    orc = Oracle()
    labels = res[0]["labels"]
    for i, (g, s) in enumerate(zip(gids, srcs)):
        assert np.array_equal(labels[i], orc.bfs(graphs[g], int(s))[0]), i
    assert len(res[0]["secs"]) == 2
    served = res[0]["served"]
    assert sum(served["per_rank_queries"]) == len(gids)
    assert served["latency_us"].shape == (len(gids),) and np.all(served["latency_us"] > 0)
    assert served["queries_per_s"] == pytest.approx(len(gids) / (served["makespan_us"] / 1e6))
