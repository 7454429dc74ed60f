"""GPU parity of the sm_100a BFS against the oracle and the reference's golden labels.

Depth labels must be bit-exact (test/bfs/test_bfs.cu:385, CompareResults);
predecessor labels must pass the reference's validity check (:389-438).
Everything goes through the C ABI of libb40c_bfs.so via the Python mirror of
b40c::graph::bfs.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_paths, load_golden

pytestmark = pytest.mark.gpu

STRATEGIES = [0, 1, 2, 3]  # expand-contract, contract-expand, two-phase, hybrid
VARIANTS = [1, 2]       # fused (persistent kernel), iterative (graph-driven per-level)


def bfs_mod():
    import back40computing_b200 as b
    return b


def expected_search_depths(strategy, g, labels):
    """GetStatistics search_depth (= iteration - 1) by strategy, derived from the
    reference's level loops: expand-contract and two-phase stop after the level
    that discovers nothing (depth d); contract-expand runs one more sweep over
    the edges of the deepest level when it has any (d + 1).  The hybrid ends in
    whichever body its last level ran, so either value is its own."""
    d = int(labels.max())
    deg = np.diff(g.row_offsets)
    ce = d + 1 if (deg[labels == d] > 0).any() else d
    return {0: {d}, 1: {ce}, 2: {d}, 3: {d, ce}}[strategy]


def run_search(g, strategy, variant, src, mark_pred=False, sizing=1.3, policy=None, problem=None,
               max_grid=0):
    b = bfs_mod()
    prob = problem or b.CsrProblem(mark_pred).from_graph(g)
    en = b.make_enactor(strategy)
    if policy:
        en.set_policy(**policy)
    b.check(prob.Reset(en.GetFrontierType(), sizing))
    rc = en.EnactSearch(prob, int(src), max_grid) if variant == 0 else (
        en.EnactFusedSearch(prob, int(src), max_grid) if variant == 1 else
        en.EnactIterativeSearch(prob, int(src), max_grid))
    b.check(rc)
    labels = prob.labels()
    stats = en.GetStatistics()
    return labels, stats


@pytest.mark.parametrize("path", golden_paths(), ids=lambda p: p.stem)
@pytest.mark.parametrize("strategy", STRATEGIES)
@pytest.mark.parametrize("variant", VARIANTS)
def test_golden_labels_bit_exact(cuda_device, path, strategy, variant):
    g, sources, golden, depths = load_golden(path)
    b = bfs_mod()
    prob = b.CsrProblem(False).from_graph(g)
    for i, s in enumerate(sources):
        labels, (_, search_depth, _) = run_search(g, strategy, variant, s, problem=prob)
        assert np.array_equal(labels, golden[i]), f"{path.stem} src {s}: first mismatch at " \
            f"{int(np.nonzero(labels != golden[i])[0][0])}"
        assert search_depth in expected_search_depths(strategy, g, golden[i])
        assert depths[i] == golden[i].max() + 1  # SimpleReferenceBfs search_depth


@pytest.mark.parametrize("path", golden_paths()[:6], ids=lambda p: p.stem)
@pytest.mark.parametrize("strategy", STRATEGIES)
@pytest.mark.parametrize("variant", VARIANTS)
def test_golden_predecessors_valid(cuda_device, oracle, path, strategy, variant):
    g, sources, golden, _ = load_golden(path)
    for i, s in enumerate(sources):
        preds, _ = run_search(g, strategy, variant, s, mark_pred=True)
        assert preds[s] == -2  # source convention (contract_expand_atomic/kernel.cuh:321-325)
        bad, reason = oracle.check_predecessors(g, preds, golden[i])
        assert bad == -1, f"{path.stem} src {s}: node {bad} fails check {reason}"
        assert np.array_equal(preds >= 0, golden[i] > 0)


@pytest.fixture(scope="module")
def rmat16():
    return bfs_mod().rmat(16, 16, seed=1)


@pytest.mark.parametrize("strategy", STRATEGIES)
@pytest.mark.parametrize("variant", [0, 1, 2])
def test_rmat16_vs_oracle(cuda_device, oracle, rmat16, strategy, variant):
    g = rmat16
    for s in g.sample_sources(3, 2):
        ref, _ = oracle.bfs(g, int(s))
        labels, _ = run_search(g, strategy, variant, s)
        assert oracle.first_mismatch(labels, ref) == -1


# Policies that route lists through every gather path: tiny thresholds push
# most lists to the CTA and grid-wide (big-list) phases; culls on and off.
POLICIES = [
    dict(cta_threads=128),
    dict(cta_threads=256),
    dict(cta_threads=512),
    dict(warp_gather_threshold=4, cta_gather_threshold=16),
    dict(warp_gather_threshold=1, cta_gather_threshold=1),
    dict(warp_gather_threshold=1000000, cta_gather_threshold=1000000),
    dict(cta_threads=512, warp_gather_threshold=8, cta_gather_threshold=600),
    dict(cull_flags=0),
    dict(cull_flags=1),
    dict(cull_flags=2),
    dict(cull_flags=3, cta_threads=128, cta_gather_threshold=100),
]


@pytest.mark.parametrize("policy", POLICIES, ids=lambda p: ",".join(f"{k}={v}" for k, v in p.items()))
@pytest.mark.parametrize("strategy", STRATEGIES)
def test_policies_rmat(cuda_device, oracle, rmat16, policy, strategy):
    g = rmat16
    s = int(g.sample_sources(1, 9)[0])
    ref, _ = oracle.bfs(g, s)
    for variant in VARIANTS:
        labels, _ = run_search(g, strategy, variant, s, policy=policy)
        assert oracle.first_mismatch(labels, ref) == -1
        preds, _ = run_search(g, strategy, variant, s, policy=policy, mark_pred=True)
        assert oracle.check_predecessors(g, preds, ref)[0] == -1


def _graph(rows, cols, n):
    return bfs_mod().from_coo(n, np.asarray(rows, np.int32), np.asarray(cols, np.int32))


EDGE_CASES = {
    "single_vertex": lambda: _graph([], [], 1),
    "isolated_source": lambda: _graph([1, 2], [2, 1], 4),
    "no_edges": lambda: _graph([], [], 50),
    "self_loops_dups": lambda: _graph([0, 0, 0, 1, 1, 2, 2, 2], [0, 1, 1, 0, 2, 2, 1, 0], 3),
    "directed_chain": lambda: _graph(list(range(999)), list(range(1, 1000)), 1000),
    "path_5000": lambda: _graph(list(range(4999)) + list(range(1, 5000)),
                                list(range(1, 5000)) + list(range(4999)), 5000),
    "star_20k": lambda: _graph([0] * 20000 + list(range(1, 20001)),
                                list(range(1, 20001)) + [0] * 20000, 20001),
}


@pytest.mark.parametrize("case", sorted(EDGE_CASES))
@pytest.mark.parametrize("strategy", STRATEGIES)
def test_edge_cases(cuda_device, oracle, case, strategy):
    g = EDGE_CASES[case]()
    for s in sorted({0, g.nodes - 1, g.nodes // 2}):
        ref, _ = oracle.bfs(g, s)
        for variant in VARIANTS:
            labels, (_, depth, _) = run_search(g, strategy, variant, s)
            assert oracle.first_mismatch(labels, ref) == -1, (case, s, variant)
            assert depth in expected_search_depths(strategy, g, ref)
            preds, _ = run_search(g, strategy, variant, s, mark_pred=True)
            assert oracle.check_predecessors(g, preds, ref)[0] == -1


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_small_grids(cuda_device, oracle, strategy):
    """A grid of 1 and 2 CTAs must give the same labels (barrier with few arrivals)."""
    g = bfs_mod().grid2d(64)
    ref, _ = oracle.bfs(g, 32 * 64 + 32)
    for grid in (1, 2, 7):
        for variant in VARIANTS:
            labels, _ = run_search(g, strategy, variant, 32 * 64 + 32, max_grid=grid)
            assert oracle.first_mismatch(labels, ref) == -1


def test_grid2d_1024_contract_expand(cuda_device, oracle):
    """The 1024x1024 lattice, source (512, 512), contract-expand (plain EnactSearch)."""
    g = bfs_mod().grid2d(1024)
    src = 512 * 1024 + 512
    ref, _ = oracle.bfs(g, src)
    for strategy in STRATEGIES:
        labels, (_, depth, _) = run_search(g, strategy, 0, src)
        assert oracle.first_mismatch(labels, ref) == -1
        assert depth in expected_search_depths(strategy, g, ref)


def test_overflow_reports_invalid_configuration(cuda_device, rmat16):
    b = bfs_mod()
    prob = b.CsrProblem(False).from_graph(rmat16)
    en = b.EnactorContractExpand()
    b.check(prob.Reset(en.GetFrontierType(), 0.001))
    rc = en.EnactSearch(prob, int(rmat16.sample_sources(1, 2)[0]))
    assert rc == b.bfs.cudaErrorInvalidConfiguration
    # Recovers after a proper reset.
    b.check(prob.Reset(en.GetFrontierType(), 1.0))
    b.check(en.EnactSearch(prob, int(rmat16.sample_sources(1, 2)[0])))


def test_barrier_timeout_is_reported_and_context_survives(cuda_device, oracle):
    b = bfs_mod()
    assert b.bfs.debug_barrier_timeout(8, 20000) == b.bfs.cudaErrorLaunchTimeout
    g = b.grid2d(32)
    ref, _ = oracle.bfs(g, 5)
    labels, _ = run_search(g, 0, 1, 5)
    assert oracle.first_mismatch(labels, ref) == -1


def test_bad_csr_rejected_on_host(cuda_device):
    b = bfs_mod()
    prob = b.CsrProblem(False)
    row = np.array([0, 1, 2], np.int32)
    assert prob.FromHostProblem(False, 2, 2, np.array([1, 5], np.int32), row, 1) == 1
    assert prob.FromHostProblem(False, 2, 2, np.array([1, 0], np.int32), np.array([0, 2, 1], np.int32), 1) == 1
    assert prob.FromHostProblem(False, 2, 2, np.array([1, 0], np.int32), row, 1) == 0


def test_source_out_of_range(cuda_device):
    b = bfs_mod()
    g = b.grid2d(8)
    prob = b.CsrProblem(False).from_graph(g)
    en = b.EnactorExpandContract()
    b.check(prob.Reset(en.GetFrontierType(), 1.3))
    assert en.EnactSearch(prob, g.nodes) == 1
    assert en.EnactSearch(prob, -1) == 1


def test_async_back_to_back(cuda_device, oracle, rmat16):
    """Searches enqueued without host syncs, each followed by its label copy."""
    b = bfs_mod()
    g = rmat16
    sources = g.sample_sources(6, 4)
    for strategy in STRATEGIES:
        prob = b.CsrProblem(False).from_graph(g)
        en = b.make_enactor(strategy)
        outs = [np.empty(g.nodes, np.int32) for _ in sources]
        for s, out in zip(sources, outs):
            b.check(prob.ResetAsync(en.GetFrontierType(), 1.3))
            b.check(en.EnactSearchAsync(prob, int(s)))
            b.check(prob.ExtractResultsAsync(out))
        b.check(en.Sync())
        for s, out in zip(sources, outs):
            ref, _ = oracle.bfs(g, int(s))
            assert oracle.first_mismatch(out, ref) == -1


@pytest.mark.parametrize("variant", [0, 2])
def test_two_label_buffers_pipeline(cuda_device, oracle, rmat16, variant):
    """Two label buffers: each Reset switches buffers and ExtractResultsAsync
    copies on a side stream while the next search runs. Every copied array
    must equal the oracle, with fused and per-level (graph) searches, the
    latter cached per buffer. Switching back to one buffer keeps the last
    search's labels."""
    b = bfs_mod()
    g = rmat16
    sources = [int(s) for s in g.sample_sources(7, 41)]
    for strategy in STRATEGIES:
        if strategy == 3 and variant == 2:
            continue  # the hybrid runs fused only
        prob = b.CsrProblem(False).from_graph(g)
        prob.set_label_buffers(2)
        en = b.make_enactor(strategy)
        outs = [np.full(g.nodes, 7, np.int32) for _ in sources]
        ptrs = set()
        for s, out in zip(sources, outs):
            b.check(prob.ResetAsync(en.GetFrontierType(), 1.3))
            ptrs.add(prob.device_pointers()["d_labels"])
            b.check(en.EnactSearchAsync(prob, s, 0, variant))
            b.check(prob.ExtractResultsAsync(out))
        b.check(en.Sync())
        b.check(prob.Sync())
        assert len(ptrs) == 2
        for s, out in zip(sources, outs):
            ref, _ = oracle.bfs(g, s)
            assert oracle.first_mismatch(out, ref) == -1, (strategy, s)
        # synchronous calls in the two-buffer mode, then back to one buffer
        ref, _ = oracle.bfs(g, sources[0])
        enact = en.EnactIterativeSearch if variant == 2 else en.EnactSearch
        b.check(prob.Reset(en.GetFrontierType(), 1.3))
        b.check(enact(prob, sources[0]))
        assert oracle.first_mismatch(prob.labels(), ref) == -1
        prob.set_label_buffers(1)
        assert oracle.first_mismatch(prob.labels(), ref) == -1
        b.check(prob.Reset(en.GetFrontierType(), 1.3))
        b.check(enact(prob, sources[1]))
        ref1, _ = oracle.bfs(g, sources[1])
        assert oracle.first_mismatch(prob.labels(), ref1) == -1
        prob.close()


def test_label_buffers_argument_check(cuda_device):
    b = bfs_mod()
    prob = b.CsrProblem(False)
    with pytest.raises(b.BfsError):
        prob.set_label_buffers(3)
    prob.close()


def test_stream_from_host(cuda_device, oracle):
    b = bfs_mod()
    g = b.rmat(12, 8, seed=3)
    s = int(g.sample_sources(1, 1)[0])
    ref, _ = oracle.bfs(g, s)
    for strategy in STRATEGIES:
        prob = b.CsrProblem(False).from_graph(g, stream_from_host=True)
        labels, _ = run_search(g, strategy, 1, s, problem=prob)
        assert oracle.first_mismatch(labels, ref) == -1


def test_problem_reused_across_strategies(cuda_device, oracle, rmat16):
    b = bfs_mod()
    g = rmat16
    prob = b.CsrProblem(False).from_graph(g)
    for s in g.sample_sources(2, 8):
        ref, _ = oracle.bfs(g, int(s))
        for strategy in [0, 1, 2, 0]:
            labels, _ = run_search(g, strategy, 1, s, problem=prob)
            assert oracle.first_mismatch(labels, ref) == -1


def test_level_log_matches_oracle_levels(cuda_device, oracle, rmat16):
    """The per-level log's frontier lengths equal the oracle's level sizes
    (expand-contract: vertex frontier of depth d at level d)."""
    b = bfs_mod()
    g = rmat16
    s = int(g.sample_sources(1, 3)[0])
    ref, _ = oracle.bfs(g, s)
    prob = b.CsrProblem(False).from_graph(g)
    for variant in VARIANTS:
        en = b.EnactorExpandContract()
        en.set_level_log(True)
        b.check(prob.Reset(en.GetFrontierType(), 1.3))
        b.check(en.EnactFusedSearch(prob, s) if variant == 1 else en.EnactIterativeSearch(prob, s))
        log = en.level_log()
        sizes = [int((ref == d).sum()) for d in range(int(ref.max()) + 1)]
        # one record per level (depths 0..d) plus the end marker
        assert len(log) == len(sizes) + 1
        assert log[0]["frontier"] + log[0]["chunks"] + log[0]["wchunks"] >= 1
        # vertices of a level are queued or, with long lists, turned into chunks
        for r, n in zip(log[:-1], sizes):
            assert r["frontier"] <= n and (r["frontier"] == n or r["chunks"] + r["wchunks"] > 0)
        assert log[-1]["frontier"] == 0 and log[-1]["chunks"] == 0 and log[-1]["wchunks"] == 0
        assert all(log[i]["start_ns"] <= log[i + 1]["start_ns"] for i in range(len(log) - 1))


def test_hybrid_switches_between_bodies(cuda_device, oracle, rmat16):
    """A small grid lowers the hybrid's saturation point (4 edges per thread), so
    most levels run as two phases; the full grid runs more of them as one
    contract-expand phase.  Labels are the same whichever body runs."""
    b = bfs_mod()
    g = rmat16
    s = int(g.sample_sources(1, 5)[0])
    ref, _ = oracle.bfs(g, s)
    d = int(ref.max())
    prob = b.CsrProblem(False).from_graph(g)
    en = b.EnactorHybrid()
    en.set_level_log(True)
    phases = {}
    for grid in (1, 16, 0):
        b.check(prob.Reset(en.GetFrontierType(), 1.3))
        b.check(en.EnactSearch(prob, s, grid))
        assert oracle.first_mismatch(prob.labels(), ref) == -1
        _, depth, _ = en.GetStatistics()
        assert depth in expected_search_depths(3, g, ref)
        phases[grid] = len(en.level_log()) - 1  # the last record marks the end
    assert phases[1] > d + 1          # two-phase levels ran
    assert phases[0] <= phases[1]     # the full grid runs at least as many levels in one phase


def _ec_search(prob, g, src, alpha, log=True):
    b = bfs_mod()
    en = b.EnactorExpandContract()
    en.set_direction_optimizing(alpha, 24 if alpha else 0)
    en.set_level_log(log)
    b.check(prob.Reset(en.GetFrontierType(), 1.0))
    b.check(en.EnactSearch(prob, int(src)))
    return prob.labels(), en.GetStatistics(), en.level_log() if log else []


@pytest.mark.parametrize("graph", ["rmat16", "er", "grid2d", "rmat_sparse"])
def test_direction_optimizing_matches_top_down(cuda_device, oracle, rmat16, graph):
    """Bottom-up levels change neither labels nor search depth nor total_queued."""
    b = bfs_mod()
    g = {"rmat16": lambda: rmat16, "er": lambda: b.erdos_renyi(20000, 24 / 19999, seed=6),
         "grid2d": lambda: b.grid2d(200), "rmat_sparse": lambda: b.rmat(15, 2, seed=9)}[graph]()
    prob = b.CsrProblem(False).from_graph(g)
    for s in g.sample_sources(3, 17):
        ref, _ = oracle.bfs(g, int(s))
        td_labels, td_stats, td_log = _ec_search(prob, g, s, 0)
        do_labels, do_stats, do_log = _ec_search(prob, g, s, 14)
        assert oracle.first_mismatch(td_labels, ref) == -1
        assert oracle.first_mismatch(do_labels, ref) == -1
        assert do_stats[1] == td_stats[1] == int(ref.max())
        assert not any(r["bottom_up"] for r in td_log)
        if graph in ("rmat16", "er"):
            assert any(r["bottom_up"] for r in do_log), do_log


def test_direction_optimizing_low_alpha_runs_most_levels_bottom_up(cuda_device, oracle, rmat16):
    """alpha = 1, beta = 1: bottom-up from the first level whose frontier edges
    exceed the unvisited edges, and it stays there."""
    b = bfs_mod()
    g = rmat16
    prob = b.CsrProblem(False).from_graph(g)
    en = b.EnactorExpandContract()
    en.set_direction_optimizing(1, 1)
    en.set_level_log(True)
    for s in g.sample_sources(4, 21):
        ref, _ = oracle.bfs(g, int(s))
        b.check(prob.Reset(en.GetFrontierType(), 1.0))
        b.check(en.EnactSearch(prob, int(s)))
        assert oracle.first_mismatch(prob.labels(), ref) == -1
        assert any(r["bottom_up"] for r in en.level_log())


@pytest.mark.parametrize("mark_pred", [False, True])
def test_direction_optimizing_after_reupload(cuda_device, oracle, mark_pred):
    """Bottom-up levels probe each vertex's heaviest neighbour, kept per graph:
    after FromHostProblem uploads another graph of the same size into the same
    problem, searches still match the oracle (a stale table would name
    non-neighbours).  grid2d has equal degrees, so its heaviest neighbour is
    often not a parent and the lists are scanned."""
    b = bfs_mod()
    graphs = [b.rmat(14, 8, seed=31), b.rmat(14, 8, seed=32), b.grid2d(128)]
    prob = b.CsrProblem(mark_pred)
    en = b.EnactorExpandContract()
    en.set_direction_optimizing(1, 1)
    en.set_level_log(True)
    for gi, g in enumerate(graphs):
        prob.from_graph(g)
        for s in g.sample_sources(2, 23):
            ref, _ = oracle.bfs(g, int(s))
            b.check(prob.Reset(en.GetFrontierType(), 1.0))
            b.check(en.EnactSearch(prob, int(s)))
            if mark_pred:
                assert oracle.check_predecessors(g, prob.labels(), ref)[0] == -1
            else:
                assert oracle.first_mismatch(prob.labels(), ref) == -1
            if gi < 2:
                assert any(r["bottom_up"] for r in en.level_log())


def test_direction_optimizing_skips_directed_graphs(cuda_device, oracle):
    """A directed graph fails the symmetry check and is searched top-down only."""
    b = bfs_mod()
    path = [p for p in golden_paths() if p.stem == "ref_random_3000_d"][0]
    g, sources, golden, _ = load_golden(path)
    prob = b.CsrProblem(False).from_graph(g)
    for i, s in enumerate(sources[:3]):
        labels, _, log = _ec_search(prob, g, s, 1)
        assert np.array_equal(labels, golden[i])
        assert not any(r["bottom_up"] for r in log)


@pytest.mark.parametrize("alpha", [1, 14])
def test_direction_optimizing_with_predecessors(cuda_device, oracle, rmat16, alpha):
    """Predecessor labels: bottom-up levels probe a copy of the visited mask and
    record the parent they find; every predecessor must be valid."""
    b = bfs_mod()
    g = rmat16
    prob = b.CsrProblem(True).from_graph(g)
    for s in g.sample_sources(3, 23):
        ref, _ = oracle.bfs(g, int(s))
        preds, _, log = _ec_search(prob, g, s, alpha)
        assert oracle.check_predecessors(g, preds, ref)[0] == -1
        assert any(r["bottom_up"] for r in log)


def test_direction_switch_arguments(cuda_device):
    b = bfs_mod()
    en = b.EnactorExpandContract()
    with pytest.raises(b.BfsError):
        en.set_direction_optimizing(14, 0)
    with pytest.raises(b.BfsError):
        en.set_direction_optimizing(-1, 24)
    with pytest.raises(b.BfsError):
        b.EnactorContractExpand().set_direction_optimizing(14, 24)
    b.EnactorContractExpand().set_direction_optimizing(0, 0)


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_instrument_statistics(cuda_device, oracle, rmat16, strategy):
    """INSTRUMENT: total_queued counts the levels' inputs and avg_duty is the
    CTAs' busy share of the longest CTA (0 < duty <= 1); labels unchanged;
    without INSTRUMENT both read 0 as in the reference."""
    b = bfs_mod()
    g = rmat16
    s = int(g.sample_sources(1, 41)[0])
    ref, _ = oracle.bfs(g, s)
    prob = b.CsrProblem(False).from_graph(g)
    for instrument in (True, False):
        en = b.make_enactor(strategy, INSTRUMENT=instrument)
        b.check(prob.Reset(en.GetFrontierType(), 1.3))
        b.check(en.EnactSearch(prob, s))
        assert oracle.first_mismatch(prob.labels(), ref) == -1
        queued, depth, duty = en.GetStatistics()
        if instrument:
            assert queued > 0
            assert 0.0 < duty <= 1.0
        else:
            assert queued == 0 and duty == 0.0


def test_eight_byte_vertex_ids(cuda_device, oracle, rmat16):
    """The g500 configuration (VertexId = long long, SizeT = int): ids are
    narrowed on upload, labels widened on extraction, results unchanged."""
    import ctypes
    from back40computing_b200._lib import lib
    b = bfs_mod()
    g = rmat16
    s = int(g.sample_sources(1, 44)[0])
    ref, _ = oracle.bfs(g, s)
    col64 = g.column_indices.astype(np.int64)
    prob = b.CsrProblem(False)
    P = ctypes.c_void_p
    assert lib().b40c_problem_from_host_ids64(prob._h, 0, g.nodes, g.edges, col64.ctypes.data_as(P),
                                              g.row_offsets.ctypes.data_as(P), 1) == 0
    en = b.make_enactor(1)
    b.check(prob.Reset(en.GetFrontierType(), 1.3))
    b.check(en.EnactSearch(prob, s))
    out = np.empty(g.nodes, np.int64)
    assert lib().b40c_problem_extract_results_ids64(prob._h, out.ctypes.data_as(P)) == 0
    assert np.array_equal(out, ref.astype(np.int64))
    bad = col64.copy()
    bad[7] = g.nodes + (1 << 33)
    assert lib().b40c_problem_from_host_ids64(prob._h, 0, g.nodes, g.edges, bad.ctypes.data_as(P),
                                              g.row_offsets.ctypes.data_as(P), 1) == 1
    assert lib().b40c_problem_from_host_ids64(prob._h, 1, g.nodes, g.edges, col64.ctypes.data_as(P),
                                              g.row_offsets.ctypes.data_as(P), 1) == 801


@pytest.mark.parametrize("strategy", [1, 2, 3])
@pytest.mark.parametrize("variant", VARIANTS)
def test_edge_frontier_total_queued_is_the_references(cuda_device, oracle, rmat16, strategy, variant):
    """Edge-frontier strategies count total_queued as the reference does: the
    sum of the levels' edge frontiers, every neighbour of every contracted
    vertex -- 1 (the source) + edges_visited -- whether a neighbour was queued,
    cut into a chunk, or dropped by the gather-time cull; labels and search
    depth unchanged."""
    b = bfs_mod()
    for g, s in ((rmat16, int(rmat16.sample_sources(1, 13)[0])), (b.grid2d(96), 48 * 96 + 48)):
        if strategy == 3 and variant == 2:
            continue  # the hybrid has one way to run
        ref, _ = oracle.bfs(g, s)
        _, edges = oracle.visit_stats(g, ref)
        prob = b.CsrProblem(False).from_graph(g)
        en = b.make_enactor(strategy, INSTRUMENT=True)
        b.check(prob.Reset(en.GetFrontierType(), 1.3))
        b.check(en.EnactFusedSearch(prob, s) if variant == 1 else en.EnactIterativeSearch(prob, s))
        assert oracle.first_mismatch(prob.labels(), ref) == -1
        queued, depth, _ = en.GetStatistics()
        assert queued == 1 + edges, (g.name, strategy, variant)
        assert depth in expected_search_depths(strategy, g, ref)


@pytest.mark.parametrize("what", [0, 1, 2])
def test_l2_persistence_keeps_labels(cuda_device, oracle, rmat16, what):
    """The persisting L2 window (visited mask, or mask and labels) changes no
    result; an out-of-range setting is rejected."""
    b = bfs_mod()
    g = rmat16
    prob = b.CsrProblem(False).from_graph(g)
    for strategy in (0, 1):
        en = b.make_enactor(strategy)
        en.set_l2_persistence(what)
        for s in g.sample_sources(2, 17 + what):
            ref, _ = oracle.bfs(g, int(s))
            b.check(prob.Reset(en.GetFrontierType(), 1.3))
            b.check(en.EnactSearch(prob, int(s)))
            assert oracle.first_mismatch(prob.labels(), ref) == -1
    with pytest.raises(b.BfsError):
        b.make_enactor(0).set_l2_persistence(3)


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_level_times_are_ordered(cuda_device, rmat16, strategy):
    """The level log's work-end time of a fused search's phase lies between the
    phase's start and the next phase's start (the grid barrier between)."""
    b = bfs_mod()
    g = rmat16
    prob = b.CsrProblem(False).from_graph(g)
    en = b.make_enactor(strategy)
    en.set_level_log(True)
    b.check(prob.Reset(en.GetFrontierType(), 1.3))
    b.check(en.EnactFusedSearch(prob, int(g.sample_sources(1, 23)[0])))
    log = en.level_log()
    assert len(log) >= 3
    for cur, nxt in zip(log[:-1], log[1:]):
        assert cur["work_end_ns"] is not None
        assert cur["start_ns"] <= cur["work_end_ns"] <= nxt["start_ns"]


@pytest.mark.parametrize("alpha", [14, 1])
def test_bottom_up_staging_matches_loads(cuda_device, oracle, rmat16, alpha):
    """Bottom-up steps with their inputs staged in shared memory by bulk copies
    and with plain loads give the oracle's labels, search depth and
    total_queued, including a graph whose vertex count is not a multiple of a
    step's 128 vertices (the last step's copies are clamped to the arrays'
    padded ends)."""
    b = bfs_mod()
    graphs = [rmat16, b.erdos_renyi(5003, 12.0 / 5002, seed=9), b.grid2d(61)]
    for g in graphs:
        prob = b.CsrProblem(False).from_graph(g)
        for s in g.sample_sources(3, 31):
            ref, _ = oracle.bfs(g, int(s))
            stats = []
            for staged in (True, False):
                en = b.EnactorExpandContract(INSTRUMENT=True)
                en.set_direction_optimizing(alpha, 24)
                en.set_bottom_up_staging(staged)
                en.set_level_log(True)
                b.check(prob.Reset(en.GetFrontierType(), 1.3))
                b.check(en.EnactSearch(prob, int(s)))
                assert oracle.first_mismatch(prob.labels(), ref) == -1, (g.name, int(s), staged)
                queued, depth, _ = en.GetStatistics()
                stats.append((queued, depth))
                if alpha == 1:
                    assert any(r["bottom_up"] for r in en.level_log()), g.name
            assert stats[0] == stats[1]
