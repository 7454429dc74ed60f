"""The N > 1 path of bench.py on CPU: two gloo ranks, as torchrun launches the
replicas on GPUs (each rank its own sources, no collective on the data path,
the slowest rank's time and the summed edges for the aggregate)."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    import bench
    import back40computing_b200 as b
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    g = b.rmat(10, 8, seed=3)
    src = [int(x) for x in bench.replica_sources(g, 8, rank)]
    # rank r "took" 10 * (r + 1) ms for 1000 * (r + 1) edges
    t, e = bench.reduce_replicas(10.0 * (rank + 1), 1000.0 * (rank + 1), world, "cpu")
    out[rank] = (src, t, e)
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_aggregate_over_gloo():
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        codes = [p.exitcode for p in procs]
        res = dict(out)
    assert codes == [0, 0], codes
    (s0, t0, e0), (s1, t1, e1) = res[0], res[1]
    assert s0 != s1                    # each replica searches its own sources
    assert t0 == t1 == 20.0            # max over ranks
    assert e0 == e1 == 3000.0          # edges summed over ranks


def test_single_replica_is_local():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.reduce_replicas(5.0, 7.0, 1, "cpu") == (5.0, 7.0)
