"""Autotuner for the search policy: CTA size, gather thresholds and the
direction switch, for single searches and for batches.

The reference fixes these at compile time per architecture (KernelPolicy,
b40c/graph/bfs/*/kernel_policy.cuh); here they are run-time settings, so the
tuner times candidate policies on the caller's own graph (or batch) with a
few sources and keeps the fastest.  Results are cached in a JSON table keyed
by a coarse graph signature (size bucket, mean degree bucket, symmetric or
not), so similar graphs reuse a tuning.

    policy = tune_enactor(graph, strategy=0)          # dict of the winning knobs
    apply_enactor_policy(enactor, policy)
    policy = tune_batch(graphs, graph_ids, sources)   # multi-search knobs
    apply_batch_policy(batch, policy)
"""
from __future__ import annotations

import itertools
import json
import math
import os
import time
from pathlib import Path
from typing import Callable, Iterable

import numpy as np

from .graphs import CsrGraph

CTA_THREADS = (128, 256, 512)
WARP_THRESHOLDS = (32, 64, 128, 256)
CTA_THRESHOLDS = (512, 1024, 4096)
DIRECTIONS = ((0, 0), (14, 24), (6, 24))  # (alpha, beta); (0, 0) = top-down only
# Narrow levels (team_ctas, max_frontier, grid_frontier), every strategy: off;
# the first levels on a 16-CTA cluster; full-grid levels of up to one edge per
# thread with the latency-first body (contract-expand and hybrid; the others
# ignore grid_frontier); both.
NARROW = ((0, 0, 0), (16, 32768, 0), (0, 0, 262144), (16, 8192, 262144), (16, 32768, 262144))
# The library's defaults for expand-contract searches and batches.
DEFAULT_POLICY = {"cta_threads": 512, "warp_gather_threshold": 128, "cta_gather_threshold": 1024,
                  "alpha": 14, "beta": 24}

DEFAULT_CACHE = Path(os.environ.get("B40C_TUNE_CACHE", Path.home() / ".cache" / "b40c_bfs_tune.json"))
# Tunings this package ships, made on a B200 by tune_enactor / tune_batch
# (the bench workloads: R-MAT s22 single searches; the 1024-search batch; every
# strategy's single searches on the lattices grid2d 1024^2 and grid3d 256^3).
SHIPPED = Path(__file__).resolve().parent / "tuned_policies.json"


def graph_signature(g: CsrGraph, symmetric: bool | None = None) -> str:
    """Coarse key: log2 of the vertex count, log2 of the mean degree (rounded),
    symmetric or not (checked on the host when not given)."""
    n, m = g.nodes, g.edges
    deg = m / max(1, n)
    if symmetric is None:
        symmetric = is_symmetric(g)
    return f"n2^{int(round(math.log2(max(n, 1))))}-d2^{int(round(math.log2(max(deg, 1e-9)))) if deg >= 1 else 0}-" \
           f"{'sym' if symmetric else 'dir'}"


def _mix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64's output function (Steele, Lea and Flood, OOPSLA 2014), wrapping uint64."""
    x = x ^ (x >> np.uint64(30))
    x = x * np.uint64(0xBF58476D1CE4E5B9)
    x = x ^ (x >> np.uint64(27))
    x = x * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def is_symmetric(g: CsrGraph, chunk: int = 1 << 24) -> bool:
    """Host check, the same test the library runs on the device: hash sums of
    (u, v) and of (v, u) over every entry agree (a graph that is not
    symmetric passes only on a 64-bit collision)."""
    row = g.row_offsets.astype(np.int64)
    col = g.column_indices
    fwd = rev = np.uint64(0)
    with np.errstate(over="ignore"):
        for lo in range(0, g.edges, chunk):
            hi = min(g.edges, lo + chunk)
            src = (np.searchsorted(row, np.arange(lo, hi), side="right") - 1).astype(np.uint64)
            dst = col[lo:hi].astype(np.uint64)
            fwd += _mix64((src << np.uint64(32)) | dst).sum(dtype=np.uint64)
            rev += _mix64((dst << np.uint64(32)) | src).sum(dtype=np.uint64)
    return bool(fwd == rev)


def candidates(strategy: int = 0, directions: bool = True) -> list[dict]:
    """Policy grid; the direction switch exists for expand-contract only."""
    dirs = DIRECTIONS if (directions and strategy == 0) else ((None, None),)
    narrow = NARROW
    out = []
    for t, w, c, (a, bb), nl in itertools.product(CTA_THREADS, WARP_THRESHOLDS, CTA_THRESHOLDS, dirs, narrow):
        if c < w:
            continue
        p = {"cta_threads": t, "warp_gather_threshold": w, "cta_gather_threshold": c}
        if a is not None:
            p["alpha"], p["beta"] = a, bb
        p["narrow"] = list(nl)
        out.append(p)
    return out


def pick_best(cands: Iterable[dict], measure: Callable[[dict], float], rounds: int = 2,
              keep: float = 0.25) -> tuple[dict, float]:
    """Successive halving: every candidate is measured once, the best `keep`
    fraction again, and so on for `rounds`; returns (best policy, its time)."""
    pool = [(c, measure(c)) for c in cands]
    for _ in range(rounds - 1):
        pool.sort(key=lambda x: x[1])
        pool = pool[:max(1, int(math.ceil(len(pool) * keep)))]
        pool = [(c, min(t, measure(c))) for c, t in pool]
    best = min(pool, key=lambda x: x[1])
    return best[0], best[1]


class TuneCache:
    """JSON table: {"<kind>/<strategy>/<signature>": {"policy": {...}, "ms": t}}.
    Entries of `seed` (read-only, e.g. SHIPPED) are used when the table at
    `path` lacks the key; new tunings are written to `path` only."""

    def __init__(self, path: Path | str | None = DEFAULT_CACHE, seed: Path | str | None = None):
        self.path = Path(path) if path else None
        self.table = {}
        for src in (seed, self.path):
            if src and Path(src).exists():
                try:
                    self.table.update(json.loads(Path(src).read_text()))
                except (OSError, json.JSONDecodeError):
                    pass

    def get(self, key: str):
        e = self.table.get(key)
        return e["policy"] if e else None

    def put(self, key: str, policy: dict, ms: float) -> None:
        self.table[key] = {"policy": policy, "ms": ms}
        if self.path:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            tmp = self.path.with_suffix(".tmp")
            tmp.write_text(json.dumps(self.table, indent=1, sort_keys=True))
            tmp.replace(self.path)


def apply_enactor_policy(enactor, policy: dict) -> None:
    enactor.set_policy(cta_threads=policy["cta_threads"], warp_gather_threshold=policy["warp_gather_threshold"],
                       cta_gather_threshold=policy["cta_gather_threshold"])
    if "alpha" in policy:
        enactor.set_direction_optimizing(policy["alpha"], policy["beta"])
    if "narrow" in policy:
        enactor.set_narrow_levels(*policy["narrow"])


def apply_batch_policy(batch, policy: dict) -> None:
    batch.set_policy(cta_threads=policy["cta_threads"], warp_gather_threshold=policy["warp_gather_threshold"],
                     cta_gather_threshold=policy["cta_gather_threshold"])
    if "alpha" in policy:
        batch.set_direction_optimizing(policy["alpha"], policy["beta"])


def tune_enactor(g: CsrGraph, strategy: int = 0, num_sources: int = 4, seed: int = 7,
                 cache: TuneCache | None = None, cands: list[dict] | None = None) -> dict:
    """Fastest policy for fused searches of `strategy` on graphs like g (device
    time of EnactSearch over a few sources)."""
    from . import bfs
    cache = cache if cache is not None else TuneCache()
    key = f"enactor/{strategy}/{graph_signature(g)}"
    hit = cache.get(key)
    if hit is not None:
        return hit
    prob = bfs.CsrProblem(False).from_graph(g)
    sources = [int(s) for s in g.sample_sources(num_sources, seed)]

    def measure(policy: dict) -> float:
        en = bfs.make_enactor(strategy)
        apply_enactor_policy(en, policy)
        total = 0.0
        for s in sources:
            bfs.check(prob.Reset(en.GetFrontierType(), 1.3))
            bfs.check(en.EnactSearch(prob, s))
            total += en.last_elapsed_ms()
        return total / len(sources)

    measure(cands[0] if cands else candidates(strategy)[0])  # warm-up (symmetry check, allocations)
    best, ms = pick_best(cands or candidates(strategy), measure)
    prob.close()
    cache.put(key, best, ms)
    return best


def tune_batch(graphs: list[CsrGraph], graph_ids, sources, cache: TuneCache | None = None,
               cands: list[dict] | None = None) -> dict:
    """Fastest multi-search policy for this mix of (graph, source) searches."""
    from .batch import BfsBatch
    cache = cache if cache is not None else TuneCache()
    sig = "+".join(sorted({graph_signature(g) for g in graphs}))
    key = f"batch/{len(graph_ids)}/{sig}"
    hit = cache.get(key)
    if hit is not None:
        return hit

    batch = BfsBatch()
    for g in graphs:
        batch.add_graph(g)

    def measure(policy: dict) -> float:
        apply_batch_policy(batch, policy)
        batch.run(graph_ids, sources, use_cuda_graph=False)  # warm-up (buffers sized for this policy)
        t = time.perf_counter()
        batch.run(graph_ids, sources, use_cuda_graph=False)
        return batch.last_elapsed_ms() or (time.perf_counter() - t) * 1e3

    best, ms = pick_best(cands or candidates(0), measure)
    batch.close()
    cache.put(key, best, ms)
    return best
