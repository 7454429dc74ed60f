"""Narrow levels (b40c_enactor_set_narrow_levels): searches of every strategy
whose small levels run on one thread-block cluster, and whose small full-grid
levels run the latency-first level body (contract-expand, hybrid), give the
oracle's labels and valid predecessors, and the same search depth and
total_queued as the plain search, whether the handover to the full grid comes
at the source, in the middle of the search, or never (two-phase searches that
end on the cluster included), and whichever body each full-grid level runs
(expand-contract with its direction switch on, as by default)."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu

CE = 1
NARROW_STRATEGIES = [0, 1, 2, 3]  # expand-contract, contract-expand, two-phase, hybrid


def bfs_mod():
    import back40computing_b200 as b
    return b


def _graphs(b):
    return [
        (b.grid2d(200), [100 * 200 + 100, 0]),
        (b.grid3d(24), [0, 12 * 24 * 24 + 12 * 24 + 12]),
        (b.rmat(15, 8, seed=4), None),
        (b.erdos_renyi(3001, 5.0 / 3000, seed=2), None),
    ]


def _search(b, prob, src, team, max_frontier, grid_frontier=0, threads=0, max_grid=0, strategy=CE):
    en = b.make_enactor(strategy, INSTRUMENT=True)
    if threads:
        en.set_policy(cta_threads=threads)
    en.set_narrow_levels(team, max_frontier, grid_frontier)
    b.check(prob.Reset(en.GetFrontierType(), 1.3))
    b.check(en.EnactSearch(prob, int(src), max_grid))
    return prob.labels(), en.GetStatistics(), en


@pytest.mark.parametrize("strategy", NARROW_STRATEGIES)
@pytest.mark.parametrize("team", [16, 8, 3, 1, 0])
def test_narrow_levels_match_oracle(cuda_device, oracle, team, strategy):
    b = bfs_mod()
    # (cluster bound, full-grid latency-first bound): handover at the source,
    # after a few levels, never; full-grid levels all tiled, all latency-first,
    # or mixed
    settings = [(0, 0), (200, 0), (1 << 24, 0), (0, 1 << 24), (200, 1 << 24), (200, 700)]
    for g, sources in _graphs(b):
        prob = b.CsrProblem(False).from_graph(g)
        srcs = sources if sources is not None else [int(s) for s in g.sample_sources(2, 41)]
        for s in srcs:
            ref, _ = oracle.bfs(g, int(s))
            _, plain_stats, _ = _search(b, prob, s, 0, 0, strategy=strategy)
            for max_frontier, grid_frontier in settings:
                labels, stats, en = _search(b, prob, s, team, max_frontier, grid_frontier, strategy=strategy)
                case = (strategy, g.name, int(s), team, max_frontier, grid_frontier)
                assert oracle.first_mismatch(labels, ref) == -1, case
                assert stats[:2] == plain_stats[:2], case
                assert (1 <= en.narrow_team() <= team) if team else en.narrow_team() == 0


@pytest.mark.parametrize("strategy", NARROW_STRATEGIES)
@pytest.mark.parametrize("max_grid", [1, 2, 5])
def test_latency_first_levels_on_small_grids(cuda_device, oracle, max_grid, strategy):
    """On a grid of a few CTAs most levels are larger than one element per
    grid thread, so they take the tiled body and the small ones the
    latency-first body, level by level: against the oracle and the plain
    search's statistics."""
    b = bfs_mod()
    for g, sources in _graphs(b):
        prob = b.CsrProblem(False).from_graph(g)
        pprob = b.CsrProblem(True).from_graph(g)
        srcs = sources if sources is not None else [int(s) for s in g.sample_sources(1, 43)]
        for s in srcs:
            ref, _ = oracle.bfs(g, int(s))
            for threads in (128, 512):
                _, plain_stats, _ = _search(b, prob, s, 0, 0, threads=threads, max_grid=max_grid, strategy=strategy)
                labels, stats, _ = _search(b, prob, s, 0, 0, 1 << 24, threads=threads, max_grid=max_grid,
                                           strategy=strategy)
                case = (strategy, g.name, int(s), max_grid, threads)
                assert oracle.first_mismatch(labels, ref) == -1, case
                assert stats[:2] == plain_stats[:2], case
                preds, _, _ = _search(b, pprob, s, 0, 0, 1 << 24, threads=threads, max_grid=max_grid,
                                      strategy=strategy)
                bad, reason = oracle.check_predecessors(g, preds, ref)
                assert bad == -1, (case, bad, reason)


@pytest.mark.parametrize("strategy", NARROW_STRATEGIES)
@pytest.mark.parametrize("threads", [128, 256, 512])
def test_narrow_levels_policies_and_predecessors(cuda_device, oracle, threads, strategy):
    b = bfs_mod()
    g = b.grid2d(128)
    src = 64 * 128 + 64
    ref, _ = oracle.bfs(g, src)
    prob = b.CsrProblem(False).from_graph(g)
    pprob = b.CsrProblem(True).from_graph(g)
    for team, max_frontier, grid_frontier in ((16, 1 << 20, 0), (0, 0, 1 << 20), (16, 100, 1 << 20)):
        labels, _, _ = _search(b, prob, src, team, max_frontier, grid_frontier, threads=threads, strategy=strategy)
        assert oracle.first_mismatch(labels, ref) == -1
        preds, _, _ = _search(b, pprob, src, team, max_frontier, grid_frontier, threads=threads, strategy=strategy)
        assert preds[src] == -2
        bad, reason = oracle.check_predecessors(g, preds, ref)
        assert bad == -1, f"node {bad} fails check {reason}"


@pytest.mark.parametrize("strategy", NARROW_STRATEGIES)
def test_narrow_levels_are_logged(cuda_device, oracle, strategy):
    """The level log of a search with narrow levels holds the same records as
    the plain search's (one per level, one per phase for two-phase: frontier,
    chunk counts, direction, end marker), the narrow ones included, each with
    its work-end time between its start and the next record's."""
    b = bfs_mod()
    g = b.grid2d(96)
    src = 48 * 96 + 48
    ref, _ = oracle.bfs(g, src)
    prob = b.CsrProblem(False).from_graph(g)
    logs = []
    for setting in ((0, 0, 0), (8, 40, 0)):  # plain; the first levels narrow, then the full grid
        en = b.make_enactor(strategy)
        en.set_narrow_levels(*setting)
        en.set_level_log(True)
        b.check(prob.Reset(en.GetFrontierType(), 1.3))
        b.check(en.EnactSearch(prob, src))
        assert oracle.first_mismatch(prob.labels(), ref) == -1
        logs.append(en.level_log())
    plain, narrow = logs
    keys = ("frontier", "chunks", "wchunks", "bottom_up")
    assert [tuple(r[k] for k in keys) for r in narrow] == [tuple(r[k] for k in keys) for r in plain]
    for cur, nxt in zip(narrow[:-1], narrow[1:]):
        assert cur["start_ns"] <= cur["work_end_ns"] <= nxt["start_ns"]


@pytest.mark.parametrize("strategy", NARROW_STRATEGIES)
@pytest.mark.parametrize("setting", [(16, 1 << 20, 0), (0, 0, 1 << 20)])
def test_narrow_levels_overflow_and_recovery(cuda_device, oracle, setting, strategy):
    b = bfs_mod()
    g = b.grid2d(256)
    src = 128 * 256 + 128
    prob = b.CsrProblem(False).from_graph(g)
    en = b.make_enactor(strategy)
    en.set_narrow_levels(*setting)
    b.check(prob.Reset(en.GetFrontierType(), 0.0005))
    assert en.EnactSearch(prob, src) == b.bfs.cudaErrorInvalidConfiguration
    ref, _ = oracle.bfs(g, src)
    b.check(prob.Reset(en.GetFrontierType(), 1.3))
    b.check(en.EnactSearch(prob, src))
    assert oracle.first_mismatch(prob.labels(), ref) == -1


def test_narrow_levels_arguments(cuda_device):
    b = bfs_mod()
    en = b.make_enactor(CE)
    for bad in ((17, 100, 0), (-1, 100, 0), (4, -1, 0), (4, 100, -1)):
        with pytest.raises(b.BfsError):
            en.set_narrow_levels(*bad)
    for strategy in NARROW_STRATEGIES:
        other = b.make_enactor(strategy)
        assert other.narrow_team() == 0  # off until set
        other.set_narrow_levels(8, 100)
        assert 1 <= other.narrow_team() <= 8


@pytest.mark.parametrize("variant", [1, 2])
def test_narrow_levels_leave_the_iterative_variant_alone(cuda_device, oracle, variant):
    """Per-level launches ignore the setting; fused searches use it."""
    b = bfs_mod()
    g = b.grid2d(80)
    src = 40 * 80 + 40
    ref, _ = oracle.bfs(g, src)
    prob = b.CsrProblem(False).from_graph(g)
    for strategy in (0, 1, 2):
        en = b.make_enactor(strategy)
        en.set_narrow_levels(16, 1 << 20, 1 << 20)
        b.check(prob.Reset(en.GetFrontierType(), 1.3))
        b.check(en.EnactFusedSearch(prob, src) if variant == 1 else en.EnactIterativeSearch(prob, src))
        assert oracle.first_mismatch(prob.labels(), ref) == -1


@pytest.mark.parametrize("alpha", [1, 14])
def test_narrow_levels_keep_the_direction_switch(cuda_device, oracle, alpha):
    """Expand-contract hands its direction-switch state to the full grid: with
    narrow levels the same levels run bottom-up as without, and labels, depth
    and total_queued are the same."""
    b = bfs_mod()
    for g in (b.rmat(15, 8, seed=4), b.grid2d(120)):
        prob = b.CsrProblem(False).from_graph(g)
        for s in g.sample_sources(3, 47):
            ref, _ = oracle.bfs(g, int(s))
            runs = []
            for setting in ((0, 0, 0), (16, 1 << 20, 0), (16, 1 << 20, 1 << 20), (4, 50, 1 << 20)):
                en = b.make_enactor(0, INSTRUMENT=True)
                en.set_direction_optimizing(alpha, 24)
                en.set_narrow_levels(*setting)
                en.set_level_log(True)
                b.check(prob.Reset(en.GetFrontierType(), 1.3))
                b.check(en.EnactSearch(prob, int(s)))
                assert oracle.first_mismatch(prob.labels(), ref) == -1, (g.name, int(s), setting)
                runs.append((en.GetStatistics()[:2], [r["bottom_up"] for r in en.level_log()]))
            assert all(r == runs[0] for r in runs), (g.name, int(s), runs)
            if alpha == 1 and g.name.startswith("rmat"):
                assert any(runs[0][1])  # the switch did fire


def test_narrow_levels_with_bottom_up_staging(cuda_device, oracle):
    """One expand-contract enactor with narrow levels on, its bottom-up
    staging switched on and off between searches (the staging changes the
    kernels' shared memory, so each configuration is checked before its first
    narrow launch): labels and statistics stay the plain search's."""
    b = bfs_mod()
    g = b.rmat(15, 8, seed=4)
    prob = b.CsrProblem(False).from_graph(g)
    en = b.make_enactor(0, INSTRUMENT=True)
    en.set_direction_optimizing(1, 24)
    en.set_narrow_levels(16, 1 << 20)
    plain = b.make_enactor(0, INSTRUMENT=True)
    plain.set_direction_optimizing(1, 24)
    for staged in (False, True, False, True):
        en.set_bottom_up_staging(staged)
        for s in g.sample_sources(2, 53):
            ref, _ = oracle.bfs(g, int(s))
            b.check(prob.Reset(plain.GetFrontierType(), 1.3))
            b.check(plain.EnactSearch(prob, int(s)))
            stats = plain.GetStatistics()[:2]
            b.check(prob.Reset(en.GetFrontierType(), 1.3))
            b.check(en.EnactSearch(prob, int(s)))
            assert oracle.first_mismatch(prob.labels(), ref) == -1, (staged, int(s))
            assert en.GetStatistics()[:2] == stats, (staged, int(s))
