"""Replica placement of batched and served BFS queries across GPUs.

One search does not shard: a level-synchronous search would exchange its
frontier between GPUs at every level.  Independent (graph, source) queries do:
every GPU holds a replica of the resident graphs, the queries are partitioned
among the GPUs, each GPU runs its share in its own multi-search launch or
request loop, and the results are gathered in one process.  Nothing crosses
GPUs on the data path; torch.distributed (NCCL between GPUs, gloo on CPU) only
carries each share's results and timings to the gathering rank.

This takes the place of the reference's multi-GPU enactor
(b40c/graph/bfs/enactor_multi_gpu.cuh:502), which splits the vertices of ONE
search over GPUs, for the batched and served paths; single searches run as
independent replicas (bench.py under torchrun).

    parts = partition(graph_ids, world, costs=edges_of_each_query)
    labels, secs = run_partitioned(graph_ids, sources, batch_share(batch), costs=...)

``run_share(indices, graph_ids, sources) -> (labels, seconds)`` is the per-rank
search: :func:`batch_share` runs a :class:`~back40computing_b200.batch.BfsBatch`
on the rank's GPU; any callable with that signature works (the tests run a
CPU search on gloo ranks to exercise the placement).
"""
from __future__ import annotations

import heapq
import time

import numpy as np


def _dist():
    try:
        import torch.distributed as dist
    except ImportError:  # pragma: no cover - torch is part of the environment
        return None
    return dist if dist.is_available() and dist.is_initialized() else None


def rank_world(group=None) -> tuple[int, int]:
    dist = _dist()
    if dist is None:
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def partition(graph_ids, world: int, costs=None, mode: str = "load") -> list[np.ndarray]:
    """Query indices of each of `world` ranks, each list in query order.

    mode "round_robin": query i goes to rank i % world.
    mode "load": longest processing time first -- queries by descending cost
    (costs[i], e.g. the edge count of query i's graph; 1 each when None), each
    to the rank with the least cost so far (ties to the lower rank).  Every
    query goes to exactly one rank."""
    n = len(graph_ids)
    if world < 1:
        raise ValueError("world must be >= 1")
    if mode == "round_robin":
        idx = np.arange(n)
        return [idx[r::world] for r in range(world)]
    if mode != "load":
        raise ValueError(f"unknown partition mode {mode!r}")
    c = np.ones(n, np.float64) if costs is None else np.asarray(costs, np.float64)
    if c.shape != (n,):
        raise ValueError("costs must hold one value per query")
    order = np.argsort(-c, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    owner = np.empty(n, np.int64)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + float(c[i]), r))
    return [np.nonzero(owner == r)[0] for r in range(world)]


def run_partitioned(graph_ids, sources, run_share, costs=None, mode: str = "load", group=None, dst: int = 0):
    """Runs this rank's share of the queries with run_share and gathers every
    share on rank dst.

    Returns, on rank dst, (labels, seconds): labels[i] = the label array of
    query i (query order), seconds[r] = rank r's time for its share; on the
    other ranks (None, None).  Every rank must call it with the same queries."""
    gids = np.ascontiguousarray(graph_ids, dtype=np.int32)
    srcs = np.ascontiguousarray(sources, dtype=np.int32)
    if gids.shape != srcs.shape:
        raise ValueError("graph_ids and sources differ in length")
    rank, world = rank_world(group)
    mine = partition(gids, world, costs, mode)[rank]
    labels, secs = run_share(mine, gids[mine], srcs[mine])
    if len(labels) != len(mine):
        raise RuntimeError("run_share returned a wrong number of label arrays")
    share = (mine.tolist(), [np.asarray(x) for x in labels], float(secs))
    dist = _dist()
    if dist is None:
        shares = [share]
    else:
        shares = [None] * world if rank == dst else None
        dist.gather_object(share, shares, dst=dst, group=group)
    if rank != dst:
        return None, None
    out = [None] * len(gids)
    for idx, labs, _ in shares:
        for i, lab in zip(idx, labs):
            if out[i] is not None:
                raise RuntimeError(f"query {i} was run by two ranks")
            out[i] = lab
    missing = [i for i, x in enumerate(out) if x is None]
    if missing:
        raise RuntimeError(f"queries {missing[:8]} were run by no rank")
    return out, [s[2] for s in shares]


def batch_share(batch, use_cuda_graph: bool = True):
    """run_share over a BfsBatch that holds every graph: one multi-search
    launch for the rank's queries; the time is the launch's device time."""

    def run(indices, gids, srcs):
        if len(indices) == 0:
            return [], 0.0
        batch.run(gids, srcs, use_cuda_graph=use_cuda_graph)
        return [batch.labels(k) for k in range(len(indices))], batch.last_elapsed_ms() / 1e3

    return run


def serve_partitioned(server, graph_ids, sources, arrival_us, costs=None, mode: str = "round_robin", group=None,
                      dst: int = 0):
    """Replays a query trace with each rank serving its share (arrival times
    kept) through its own BfsServer, which holds every graph.

    Returns on rank dst {"queries_per_s", "p50_us", "p99_us", "latency_us"
    (query order), "makespan_us" (the slowest rank's), "per_rank_queries"};
    None on the other ranks."""
    gids = np.ascontiguousarray(graph_ids, dtype=np.int32)
    srcs = np.ascontiguousarray(sources, dtype=np.int32)
    arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
    rank, world = rank_world(group)
    mine = partition(gids, world, costs, mode)[rank]
    if len(mine):
        lat, span = server.run_trace(gids[mine], srcs[mine], arr[mine] - arr[mine].min())
    else:
        lat, span = np.zeros(0), 0.0
    share = (mine.tolist(), np.asarray(lat).tolist(), float(span))
    dist = _dist()
    if dist is None:
        shares = [share]
    else:
        shares = [None] * world if rank == dst else None
        dist.gather_object(share, shares, dst=dst, group=group)
    if rank != dst:
        return None
    lat_all = np.zeros(len(gids))
    for idx, lat_r, _ in shares:
        lat_all[np.asarray(idx, dtype=np.int64)] = lat_r
    span = max(s[2] for s in shares)
    return {"queries_per_s": len(gids) / (span / 1e6) if span > 0 else float("inf"),
            "p50_us": float(np.percentile(lat_all, 50)) if len(gids) else 0.0,
            "p99_us": float(np.percentile(lat_all, 99)) if len(gids) else 0.0,
            "latency_us": lat_all, "makespan_us": span, "per_rank_queries": [len(s[0]) for s in shares]}


def wall_share(search):
    """run_share from a per-query search callable search(graph_id, source) ->
    labels, timed on the host clock (for CPU searches)."""

    def run(indices, gids, srcs):
        t0 = time.perf_counter()
        labels = [search(int(g), int(s)) for g, s in zip(gids, srcs)]
        return labels, time.perf_counter() - t0

    return run
