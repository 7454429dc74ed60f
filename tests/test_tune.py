"""Autotuner: candidate grid, successive halving, cache, and (on a GPU) that
the tuned policies give the oracle's labels."""
from __future__ import annotations

import numpy as np
import pytest


def test_candidates_cover_the_knobs():
    from back40computing_b200 import tune
    ec = tune.candidates(0)
    assert {c["cta_threads"] for c in ec} == set(tune.CTA_THREADS)
    assert {c["warp_gather_threshold"] for c in ec} == set(tune.WARP_THRESHOLDS)
    assert {(c["alpha"], c["beta"]) for c in ec} == set(tune.DIRECTIONS)
    assert all("alpha" not in c for c in tune.candidates(1))  # no direction switch off expand-contract
    assert all(c["cta_gather_threshold"] >= c["warp_gather_threshold"] for c in ec)
    # narrow levels: every strategy, every setting with every other knob
    base = len([1 for t in tune.CTA_THREADS for w in tune.WARP_THRESHOLDS for c in tune.CTA_THRESHOLDS if c >= w])
    for strategy in (0, 1, 2, 3):
        cs = tune.candidates(strategy)
        assert {tuple(c["narrow"]) for c in cs} == set(tune.NARROW)
        dirs = len(tune.DIRECTIONS) if strategy == 0 else 1
        assert len(cs) == base * len(tune.NARROW) * dirs


def test_apply_enactor_policy_sets_every_knob():
    from back40computing_b200 import tune

    class Rec:
        def __init__(self):
            self.calls = []

        def __getattr__(self, name):
            return lambda *a, **k: self.calls.append((name, a, k))

    r = Rec()
    tune.apply_enactor_policy(r, {"cta_threads": 512, "warp_gather_threshold": 128, "cta_gather_threshold": 4096,
                                  "narrow": [16, 8192, 262144]})
    assert ("set_narrow_levels", (16, 8192, 262144), {}) in r.calls
    assert [c[0] for c in r.calls] == ["set_policy", "set_narrow_levels"]


def test_successive_halving_finds_the_minimum():
    from back40computing_b200 import tune
    cands = [{"k": i} for i in range(40)]
    calls = []

    def measure(c):
        calls.append(c["k"])
        return abs(c["k"] - 17) + 1.0

    best, t = tune.pick_best(cands, measure, rounds=3, keep=0.25)
    assert best["k"] == 17 and t == 1.0
    assert len(calls) < 40 * 3  # later rounds measure only the leaders


def test_shipped_table_is_well_formed():
    """The shipped tunings: keys of the cache's form, knobs within the ranges
    the library's setters accept (checked here, without a GPU)."""
    import json
    from back40computing_b200 import tune
    table = json.loads(tune.SHIPPED.read_text())
    assert table
    for key, entry in table.items():
        kind, rest = key.split("/", 1)
        assert kind in ("enactor", "batch"), key
        pol, ms = entry["policy"], entry["ms"]
        assert ms > 0
        assert pol["cta_threads"] in tune.CTA_THREADS
        assert pol["warp_gather_threshold"] in tune.WARP_THRESHOLDS
        assert pol["cta_gather_threshold"] in tune.CTA_THRESHOLDS
        if kind == "enactor":
            strategy, sig = rest.split("/", 1)
            assert int(strategy) in (0, 1, 2, 3) and sig.startswith("n2^"), key
            if "alpha" in pol:
                assert int(strategy) == 0 and (pol["alpha"], pol["beta"]) in tune.DIRECTIONS, key
            if "narrow" in pol:
                team, max_frontier, grid_frontier = pol["narrow"]
                assert 0 <= team <= 16 and max_frontier >= 0 and grid_frontier >= 0, key


def test_cache_round_trip(tmp_path):
    from back40computing_b200 import tune
    path = tmp_path / "tune.json"
    c = tune.TuneCache(path)
    c.put("enactor/0/x", {"cta_threads": 256}, 1.5)
    assert tune.TuneCache(path).get("enactor/0/x") == {"cta_threads": 256}
    assert tune.TuneCache(path).get("enactor/0/y") is None


def test_graph_signature_and_symmetry():
    import back40computing_b200 as b
    from back40computing_b200 import tune
    g = b.rmat(10, 8, seed=2)
    assert tune.is_symmetric(g)
    d = b.from_coo(4, [0, 1, 2], [1, 2, 3])
    assert not tune.is_symmetric(d)
    assert tune.graph_signature(g).endswith("sym") and tune.graph_signature(d).endswith("dir")


@pytest.mark.gpu
def test_tuned_policies_keep_labels(cuda_device, oracle):
    import back40computing_b200 as b
    from back40computing_b200 import tune
    from back40computing_b200.batch import BfsBatch
    g = b.rmat(13, 16, seed=8)
    cache = tune.TuneCache(None)
    small = tune.candidates(0)[::9]
    pol = tune.tune_enactor(g, 0, num_sources=2, cache=cache, cands=small)
    assert pol in small and cache.get(f"enactor/0/{tune.graph_signature(g)}") == pol
    en = b.make_enactor(0)
    tune.apply_enactor_policy(en, pol)
    prob = b.CsrProblem(False).from_graph(g)
    s = int(g.sample_sources(1, 3)[0])
    b.check(prob.Reset(en.GetFrontierType(), 1.3))
    b.check(en.EnactSearch(prob, s))
    assert oracle.first_mismatch(prob.labels(), oracle.bfs(g, s)[0]) == -1

    graphs = [g, b.grid2d(48)]
    gids = [0, 1, 0, 1]
    srcs = [int(graphs[k].sample_sources(1, 5 + i)[0]) for i, k in enumerate(gids)]
    bpol = tune.tune_batch(graphs, gids, srcs, cache=cache, cands=small)
    batch = BfsBatch()
    tune.apply_batch_policy(batch, bpol)
    for gg in graphs:
        batch.add_graph(gg)
    batch.run(gids, srcs)
    for i, (k, s) in enumerate(zip(gids, srcs)):
        assert oracle.first_mismatch(batch.labels(i), oracle.bfs(graphs[k], s)[0]) == -1


@pytest.mark.gpu
def test_shipped_policies_keep_labels(cuda_device, oracle):
    """Every single-search policy the package ships (tuned on a B200 for the
    bench graphs), applied to small graphs of each kind: the oracle's labels."""
    import json
    import back40computing_b200 as b
    from back40computing_b200 import tune
    table = json.loads(tune.SHIPPED.read_text())
    graphs = [(b.grid2d(100), 50 * 100 + 50), (b.grid3d(20), 0), (b.rmat(12, 16, seed=3), None)]
    refs = []
    for g, s in graphs:
        s = int(g.sample_sources(1, 9)[0]) if s is None else s
        refs.append((g, s, oracle.bfs(g, s)[0], b.CsrProblem(False).from_graph(g), b.CsrProblem(True).from_graph(g)))
    keys = [k for k in table if k.startswith("enactor/")]
    assert keys
    for key in keys:
        strategy = int(key.split("/")[1])
        en = b.make_enactor(strategy)
        tune.apply_enactor_policy(en, table[key]["policy"])
        for g, s, ref, prob, pprob in refs:
            b.check(prob.Reset(en.GetFrontierType(), 1.3))
            b.check(en.EnactSearch(prob, s))
            assert oracle.first_mismatch(prob.labels(), ref) == -1, (key, g.name)
            b.check(pprob.Reset(en.GetFrontierType(), 1.3))
            b.check(en.EnactSearch(pprob, s))
            bad, reason = oracle.check_predecessors(g, pprob.labels(), ref)
            assert bad == -1, (key, g.name, bad, reason)
