"""Benchmark of the B200 BFS on the R-MAT scale-22 workload.

Workload (default): R-MAT scale 22, edge factor 16, a/b/c/d = .57/.19/.19/.05,
self-loops removed, duplicates kept, symmetrized (~134M int32 CSR entries);
64 sources drawn with seed 2 among vertices of degree > 0.  Synthetic, seeded.

A step is one BFS from each of the 64 sources (Reset + EnactSearch each).  The
headline strategy is expand-contract (fused persistent kernel); contract-expand,
two-phase and hybrid are timed the same way and reported under "strategies".

  value   GTEPS = sum of edges_visited over the step's searches / device time,
          CSR resident in HBM, CUDA events on the enactor's stream.
  e2e     same metric through the public API with host buffers: every step
          uploads the CSR from pinned host memory (FromHostProblem), runs the 64
          searches and copies each label array back to pinned host memory.
          Steps alternate two CsrProblems (each with its own enactor and stream),
          so one step's upload overlaps the previous step's searches and copies.
  roofline  algorithmic bytes per search, 4E + 20V (column indices read once,
          a row-offset pair, a label write, a frontier write and read per
          visited vertex) / the fused kernel's average duration, against the
          measured HBM copy bandwidth.

  batched   1024 searches over 64 graphs (R-MAT scale 12..20, Erdos-Renyi) in
          one multi-search launch vs the same searches as back-to-back
          EnactSearch calls; queries/s, every label array checked.
  served    Poisson traces (1K, 10K, 50K req/s, and all at once) over 32
          resident graphs through the continuous-batching server; queries/s
          and p50/p99 latency against sequential EnactSearch serving the
          same trace.

  lattices  grid2d 1024^2 and grid3d 256^3 single searches, every strategy
          (deep, narrow searches: per-level cost rather than bandwidth).

--impl reference runs the reference's own CPU BFS (SimpleReferenceBfs, built
into oracle/_ref) on all host cores instead.  With torchrun each rank runs an
independent replica (its own 64 sources; no collective on the data path) and
rank 0 prints the aggregate over the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GTEPS (R-MAT s22 BFS)"
UNIT = "GTEPS"
NUM_SOURCES = 64
STRATEGY_NAMES = {0: "expand_contract", 1: "contract_expand", 2: "two_phase", 3: "hybrid"}
HEADLINE = 0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--strategies", default="0,1,2,3")
    ap.add_argument("--variant", type=int, default=1, help="1 fused, 2 iterative (graph-driven)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 1024-search batched leg")
    ap.add_argument("--no-served", action="store_true", help="skip the Poisson-trace serving leg")
    ap.add_argument("--no-lattices", action="store_true", help="skip the grid2d / grid3d single-search leg")
    ap.add_argument("--batched-max-scale", type=int, default=20, help="largest R-MAT scale of the batched set")
    ap.add_argument("--batched-policy", default="tuned", choices=["tuned", "default"],
                    help="autotuned multi-search policy, or the library defaults")
    ap.add_argument("--verify", type=int, default=-1,
                    help="sources of each strategy checked against the oracle during warm-up (-1: all)")
    ap.add_argument("--sources", type=int, default=NUM_SOURCES, help="sources per step (64 for the bench line)")
    return ap.parse_args()


def dist_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_sources(g, count, rank):
    """Sources of one replica: each rank searches its own seeded sample."""
    return g.sample_sources(count, 2 + 1000 * rank)


def reduce_replicas(local_time, local_edges, world, device):
    """(max time over ranks, edges summed over ranks): the replicas' aggregate
    throughput is the total edges over the slowest rank's time."""
    if world == 1:
        return float(local_time), float(local_edges)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local_time)], dtype=torch.float64, device=device)
    e = torch.tensor([float(local_edges)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), float(e.item())


def make_graph(scale, ef):
    from back40computing_b200 import graphs
    return graphs.rmat(scale, ef, 0.57, 0.19, 0.19, seed=1, undirected=True)


def bench_config(args, nodes, edges, nsrc, world):
    """The workload both arms report (identical dicts, so the two lines compare)."""
    return {"workload": f"BFS rmat-s{args.scale}-ef{args.edge_factor} (a=.57 b=.19 c=.19, seed 1, symmetrized), "
                        f"{nsrc} sources/step (seed 2)",
            "nodes": int(nodes), "edges": int(edges), "parallelism": f"replicas x{world}",
            "l2": ("inputs larger than L2" if 4 * edges > 126e6 else "inputs smaller than L2")
                  + " (column indices %.0f MB)" % (4 * edges / 1e6)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_traffic(scale, strategy):
    """DRAM bytes (read + write) of one launch of a strategy's fused kernel on
    this workload, from the committed ncu capture (profiles/dram_fused_rmat22.md,
    lines "traffic_bytes_<strategy>: <bytes>"); None when not captured."""
    prof = ROOT / "profiles" / "dram_fused_rmat22.md"
    if scale != 22 or not prof.exists():
        return None
    key = f"traffic_bytes_{STRATEGY_NAMES[strategy]}:"
    for line in prof.read_text().splitlines():
        if line.startswith(key):
            return float(line.split(":", 1)[1])
    return None


class ClockSampler:
    """SM clock and throttle reasons sampled in the background during a timed
    region: every 10 ms through NVML (reads only), else every 200 ms through
    nvidia-smi."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.samples = []  # (sm_mhz, max_mhz, reasons)
        self.thread = None
        self.stop_flag = threading.Event()
        self.nvml = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._poll_nvml, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _poll_nvml(self):
        nv = self.nvml
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)
                active = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                reasons = [name for name, attr in self.REASONS if active & getattr(nv, attr, 0)]
                self.samples.append((float(sm), float(self.max_mhz), reasons))
            except Exception:
                pass
            self.stop_flag.wait(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_flag.set()
            self.thread.join(timeout=2)
        elif self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)
            names = [n for n, _ in self.REASONS]
            for ln in self.lines:
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm, mx = float(parts[1]), float(parts[2])
                except ValueError:
                    continue
                self.samples.append((sm, mx, [n for n, v in zip(names, parts[5:9]) if v.lower() == "active"]))
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm = [x[0] for x in self.samples]
        reasons = sorted({r for x in self.samples for r in x[2]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(x[1] for x in self.samples) if sm else None,
                "reasons": reasons, "samples": len(sm), "source": "nvml" if self.nvml is not None else "nvidia-smi"}


# ------------------------------------------------------------------------------------------
# Reference arm: the reference's CPU BFS on the host cores
# ------------------------------------------------------------------------------------------

def cpu_engine():
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle, ReferenceBfs
    if ReferenceBfs.available():
        return ReferenceBfs(), "reference"
    return Oracle(), "port"


def run_cpu(g, sources, threads):
    """Independent searches over `threads` host threads; returns (edges, seconds)."""
    eng, kind = cpu_engine()
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    sys.stdout.flush()
    os.dup2(devnull, 1)  # the reference prints per search
    try:
        t0 = time.perf_counter()
        ev = eng.bfs_many(g, sources, threads)
        dt = time.perf_counter() - t0
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    return int(ev.sum()), dt, kind


def reference_arm(args):
    """The reference's own CPU BFS (SimpleReferenceBfs from oracle/_ref, or the
    oracle's restatement when it is absent) on every host thread, over the same
    graph and the same 64 sources per step as the GPU arm.  The graph comes
    from the oracle's restated generator, so this arm never loads the product
    library."""
    rank, world, _ = dist_info()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import rmat as oracle_rmat
    g = oracle_rmat(args.scale, args.edge_factor, 0.57, 0.19, 0.19, seed=1, undirected=True)
    sources = g.sample_sources(args.sources, 2)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        run_cpu(g, sources, threads)
    edges, secs = 0, 0.0
    kind = "port"
    for _ in range(args.steps):
        e, dt, kind = run_cpu(g, sources, threads)
        edges += e
        secs += dt
    gteps = edges / secs / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": gteps, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded R-MAT, 64 sources)",
        "config": bench_config(args, g.nodes, g.edges, len(sources), args.gpus),
        "cpu_baseline": {"value": gteps, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"all {len(sources)} sources per step x {args.steps} steps, "
                                   f"one search at a time per host thread"},
        "e2e": {"value": gteps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "graph_sha256": g.sha256(),
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# Batched and served legs (multi-search kernel vs back-to-back single searches)
# ------------------------------------------------------------------------------------------

def batched_set(seed=4, max_scale=20):
    """64 graphs: R-MAT with scale uniform in 12..max_scale (20 for the bench
    line) and edge factor uniform in 8..32, every fourth an Erdos-Renyi
    G(n, 16/(n-1)) of the same n; 16 seeded sources each (1024 searches)."""
    from back40computing_b200 import graphs
    rng = np.random.default_rng(seed)
    gs, desc = [], []
    for i in range(64):
        scale = min(int(rng.integers(12, 21)), max_scale)
        ef = int(rng.integers(8, 33))
        n = 1 << scale
        if i % 4 == 3:
            gs.append(graphs.erdos_renyi(n, 16.0 / (n - 1), seed=100 + i))
            desc.append(f"er-{scale}")
        else:
            gs.append(graphs.rmat(scale, ef, seed=100 + i, undirected=True))
            desc.append(f"rmat-{scale}-{ef}")
    gids = np.repeat(np.arange(64, dtype=np.int32), 16)
    srcs = np.concatenate([g.sample_sources(16, 200 + i) for i, g in enumerate(gs)]).astype(np.int32)
    return gs, desc, gids, srcs


def served_set(main_graph):
    """32 resident graphs: 24 R-MAT (scales 14..22, edge factor 16; the scale-22
    one is the headline graph) and 8 grids of 64K..16M vertices."""
    from back40computing_b200 import graphs
    gs, desc = [], []
    scales = [14, 15, 16, 17, 18, 19, 20, 21, 14, 15, 16, 17, 18, 19, 20, 14, 15, 16, 17, 18, 19, 14, 16, 22]
    for i, sc in enumerate(scales):
        if sc == 22:
            gs.append(main_graph)
        else:
            gs.append(graphs.rmat(sc, 16, seed=300 + i, undirected=True))
        desc.append(f"rmat-{sc}")
    for w in (256, 512, 1024, 2048):
        gs.append(graphs.grid2d(w))
        desc.append(f"grid2d-{w}")
    for w in (40, 64, 128, 256):
        gs.append(graphs.grid3d(w))
        desc.append(f"grid3d-{w}")
    return gs, desc


def _crc(a):
    import zlib
    return zlib.crc32(np.ascontiguousarray(a).view(np.uint8))


class SequentialSearches:
    """Back-to-back plain single searches (Reset + EnactSearch on the
    expand-contract enactor), one resident CsrProblem per graph."""

    def __init__(self, b, gs, stream):
        self.b = b
        self.stream = stream
        self.problems = []
        for g in gs:
            p = b.CsrProblem(False).from_graph(g)
            p.set_stream(stream.cuda_stream)
            self.problems.append(p)
        self.en = b.make_enactor(HEADLINE)
        self.en.set_stream(stream.cuda_stream)
        self.ft = self.en.GetFrontierType()

    def enqueue(self, gid, src):
        b = self.b
        b.check(self.problems[gid].ResetAsync(self.ft, 1.3))
        b.check(self.en.EnactSearchAsync(self.problems[gid], int(src), 0, 1))

    def run(self, gid, src):
        """One synchronous query: Reset + EnactSearch, waiting for the search."""
        b = self.b
        b.check(self.problems[gid].Reset(self.ft, 1.3))
        b.check(self.en.EnactSearch(self.problems[gid], int(src)))

    def labels(self, gid):
        b = self.b
        b.check(self.en.Sync())
        return self.problems[gid].labels()

    def close(self):
        for p in self.problems:
            p.close()
        self.problems = []
        del self.en


def batched_leg(b, torch, stream, args):
    """1024 searches over 64 graphs: one batched launch (CUDA graph replay) vs
    the same searches as back-to-back EnactSearch calls; device time, labels
    compared by checksum for every search."""
    from back40computing_b200.batch import BfsBatch
    gs, desc, gids, srcs = batched_set(max_scale=args.batched_max_scale)
    n = len(gids)
    # crc32 of the oracle's labels of every search.
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle
    orc = Oracle()
    crc_ref = np.zeros(n, np.int64)
    for gi, g in enumerate(gs):
        idx = np.nonzero(gids == gi)[0]
        refs, _ = orc.bfs_many_labels(g, srcs[idx])
        for k, i in enumerate(idx):
            crc_ref[i] = _crc(refs[k])
        del refs
    seq = SequentialSearches(b, gs, stream)
    crc_seq = np.zeros(n, np.int64)
    edges = np.zeros(n, np.int64)
    degs = [g.degrees().astype(np.int64) for g in gs]
    for i in range(n):
        seq.enqueue(gids[i], srcs[i])
        lab = seq.labels(gids[i])
        crc_seq[i] = _crc(lab)
        edges[i] = int(degs[gids[i]][lab > -1].sum())
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def time_seq():
        ev[0].record(stream)
        for i in range(n):
            seq.enqueue(gids[i], srcs[i])
        ev[1].record(stream)
        b.check(seq.en.Sync())
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1])

    bad = np.nonzero(crc_seq != crc_ref)[0]
    if bad.size:
        raise SystemExit(f"bench: single-search labels differ from the oracle for searches {bad[:8].tolist()}")
    for _ in range(args.warmup):
        time_seq()
    seq_ms = [time_seq() for _ in range(args.steps)]
    seq.close()

    # The multi-search policy picked by the autotuner for this workload (its
    # B200 result ships with the package; a different workload is tuned here).
    from back40computing_b200 import tune
    policy = (tune.tune_batch(gs, gids, srcs, cache=tune.TuneCache(None, seed=tune.SHIPPED))
              if args.batched_policy == "tuned" else dict(tune.DEFAULT_POLICY))
    batch = BfsBatch()
    tune.apply_batch_policy(batch, policy)
    batch.set_stream(stream.cuda_stream)
    for g in gs:
        batch.add_graph(g)
    batch.run(gids, srcs, use_cuda_graph=True)
    mismatched = [i for i in range(n) if _crc(batch.labels(i)) != crc_ref[i]]
    if mismatched:
        raise SystemExit(f"bench: batched labels differ from the oracle for searches {mismatched[:8]}")
    for _ in range(args.warmup):
        batch.run(gids, srcs, use_cuda_graph=True)
    bat_ms = []
    for _ in range(args.steps):
        batch.run(gids, srcs, use_cuda_graph=True)
        bat_ms.append(batch.last_elapsed_ms())
    batch.close()
    s_ms, b_ms = float(np.median(seq_ms)), float(np.median(bat_ms))
    return {
        "workload": f"64 graphs (48 R-MAT scale 12..{args.batched_max_scale} ef 8..32, 16 Erdos-Renyi mean degree 16), "
                    "16 sources each",
        "searches": n, "graph_edges_total": int(sum(g.edges for g in gs)),
        "queries_per_s": n / (b_ms / 1e3), "gteps": float(edges.sum()) / (b_ms / 1e3) / 1e9,
        "ms_per_batch": b_ms,
        "sequential_queries_per_s": n / (s_ms / 1e3), "sequential_ms": s_ms,
        "speedup_vs_sequential": s_ms / b_ms,
        "policy": policy,
        "labels": "every search's labels equal the oracle's (crc32 of all %d label arrays, batched and "
                  "single searches)" % n,
        "timing": "device time, median of %d; sequential = back-to-back async Reset+EnactSearch" % args.steps,
    }


def lattice_leg(b, torch, stream, args):
    """The lattice workloads: grid2d 1024 x 1024 from its centre (1,048,576
    vertices, 4,190,208 entries) and grid3d 256^3 from vertex 0 (16,777,216
    vertices, 100,270,080 entries; 766 levels): single searches with each
    strategy in the persistent kernel (with the autotuner's policy for the
    graph, and with the library defaults) and as per-level launches, device
    time, labels checked against the oracle once."""
    from back40computing_b200 import graphs, tune
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle
    orc = Oracle()
    out = {}
    for name, g, src in (("grid2d-1024", graphs.grid2d(1024), 512 * 1024 + 512), ("grid3d-256", graphs.grid3d(256), 0)):
        ref, _ = orc.bfs(g, src)
        E = float(g.degrees()[ref > -1].astype(np.int64).sum())
        prob = b.CsrProblem(False).from_graph(g)
        prob.set_stream(stream.cuda_stream)
        row = {"nodes": g.nodes, "edges": g.edges, "source": src, "depth": int(ref.max())}
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        def fused_ms(en):
            ft = en.GetFrontierType()
            b.check(prob.Reset(ft, 1.3))
            b.check(en.EnactSearch(prob, src))
            if orc.first_mismatch(prob.labels(), ref) != -1:
                raise SystemExit(f"bench: {name} labels of strategy {strat} differ from the oracle")
            ms = []
            for _ in range(max(3, args.steps // 2)):
                b.check(prob.ResetAsync(ft, 1.3))
                ev[0].record(stream)
                b.check(en.EnactSearchAsync(prob, src, 0, 1))
                ev[1].record(stream)
                b.check(en.Sync())
                ms.append(ev[0].elapsed_time(ev[1]))
            return float(np.median(ms))

        for strat in (0, 1, 2, 3):
            en = b.make_enactor(strat)
            en.set_stream(stream.cuda_stream)
            ft = en.GetFrontierType()
            t_default = fused_ms(en)
            # The autotuner's policy for this graph (its B200 result ships with
            # the package; a graph it has not seen is tuned here).
            policy = tune.tune_enactor(g, strat, cache=tune.TuneCache(None, seed=tune.SHIPPED))
            tuned = b.make_enactor(strat)
            tuned.set_stream(stream.cuda_stream)
            tune.apply_enactor_policy(tuned, policy)
            t = fused_ms(tuned)
            del tuned
            row[STRATEGY_NAMES[strat]] = {"ms": t, "gteps": E / (t / 1e3) / 1e9, "us_per_level": t * 1e3 / (row["depth"] + 1),
                                          "policy": policy, "default_policy_ms": t_default}
            if strat != 3:  # the same search as per-level launches (a CUDA graph with a conditional loop)
                it_ms = []
                for _ in range(3):
                    b.check(prob.ResetAsync(ft, 1.3))
                    ev[0].record(stream)
                    b.check(en.EnactSearchAsync(prob, src, 0, 2))
                    ev[1].record(stream)
                    b.check(en.Sync())
                    it_ms.append(ev[0].elapsed_time(ev[1]))
                row[STRATEGY_NAMES[strat]]["per_level_launches_ms"] = float(np.median(it_ms[1:]))
            del en
        prob.close()
        out[name] = row
    return out


def served_leg(b, torch, stream, args, main_graph):
    """Poisson traces over 32 resident graphs through the continuous-batching
    server, against sequential plain EnactSearch serving the same trace in FIFO
    order (each query's measured device service time)."""
    from back40computing_b200.serve import BfsServer, poisson_arrivals
    gs, desc = served_set(main_graph)
    G = len(gs)
    pool = [g.sample_sources(16, 400 + i) for i, g in enumerate(gs)]
    # Every (graph, source) pair searched alone: the labels each served query must reproduce.
    seq = SequentialSearches(b, gs, stream)
    crc = np.zeros((G, 16), np.int64)
    for gi in range(G):
        for k, s in enumerate(pool[gi]):
            seq.enqueue(gi, s)
            crc[gi, k] = _crc(seq.labels(gi))
    budget = min(48 << 30, int(torch.cuda.mem_get_info()[0] * 0.6))
    srv = BfsServer(max_slots=1024, hbm_budget_bytes=budget)
    for g in gs:
        srv.add_graph(g)

    def trace(nq, rate, seed):
        rng = np.random.default_rng(seed)
        gids = rng.integers(0, G, nq).astype(np.int32)
        ks = rng.integers(0, 16, nq)
        srcs = np.array([pool[g][k] for g, k in zip(gids, ks)], np.int32)
        arr = np.zeros(nq) if rate is None else poisson_arrivals(nq, rate, seed)
        return gids, ks, srcs, arr

    # Identity: a mixed trace with labels kept, every query against its lone search.
    gids, ks, srcs, arr = trace(256, 50000.0, 11)
    _, _, labs = srv.run_trace(gids, srcs, arr, keep_labels=True)
    bad = [i for i in range(len(gids)) if _crc(labs[i]) != crc[gids[i], ks[i]]]
    if bad:
        raise SystemExit(f"bench: served labels differ from lone searches for queries {bad[:8]}")
    del labs
    out = {"workload": "32 resident graphs (24 R-MAT scale 14..22 ef 16, grid2d 256..2048, grid3d 40..256), "
                       "queries (graph, source) uniform over graphs, 16 seeded sources per graph",
           "labels": "identical alone and in the mix (crc32, 256-query trace at 50K req/s)"}
    rates = []
    traces = []
    for rate, nq in ((1000.0, 1000), (10000.0, 2000), (50000.0, 4000), (None, 4000)):
        gids, ks, srcs, arr = trace(nq, rate, 21 + nq)
        traces.append((rate, nq, gids, srcs, arr))
        lat, span = srv.run_trace(gids, srcs, arr)
        rates.append({
            "rate_per_s": rate if rate is not None else "all at t=0", "queries": nq,
            "queries_per_s": nq / (span / 1e6), "p50_us": float(np.percentile(lat, 50)),
            "p99_us": float(np.percentile(lat, 99))})
    st = srv.stats()
    srv.close()
    # The same traces served sequentially, for real: one query at a time in
    # arrival order through the plain synchronous Reset + EnactSearch,
    # latency = completion - arrival on the host clock.
    for r, (rate, nq, gids, srcs, arr) in zip(rates, traces):
        fin = np.zeros(nq)
        t0 = time.perf_counter()
        for i in range(nq):
            now = (time.perf_counter() - t0) * 1e6
            if arr[i] > now:
                time.sleep((arr[i] - now) / 1e6)
            seq.run(gids[i], srcs[i])
            fin[i] = (time.perf_counter() - t0) * 1e6
        slat = fin - arr
        r.update({"sequential_queries_per_s": nq / (fin[-1] / 1e6),
                  "sequential_p50_us": float(np.percentile(slat, 50)),
                  "sequential_p99_us": float(np.percentile(slat, 99))})
    seq.close()
    sat = rates[-1]
    out.update({"rates": rates, "saturated_queries_per_s": sat["queries_per_s"],
                "sequential_saturated_queries_per_s": sat["sequential_queries_per_s"],
                "speedup_vs_sequential": sat["queries_per_s"] / sat["sequential_queries_per_s"],
                "server": st,
                "timing": "server: host clock in the request loop, real-time replay; sequential: the same "
                          "traces replayed in real time through synchronous Reset + EnactSearch, one query at a "
                          "time in arrival order, host clock"})
    return out


def summary_block(e2e, batched, served, lattices, results):
    """The line's figures in a few keys placed near its front (the full
    objects follow later in the line)."""
    out = {"strategies_ms": {STRATEGY_NAMES[s]: round(r["kernel_ms_mean"], 4) for s, r in results.items()}}
    if e2e:
        out["e2e_gteps"] = round(e2e["value"], 1)
    if batched:
        out["batched_queries_per_s"] = round(batched["queries_per_s"])
        out["batched_speedup_vs_sequential"] = round(batched["speedup_vs_sequential"], 2)
    if served:
        out["served_queries_per_s"] = round(served["saturated_queries_per_s"])
        out["served_speedup_vs_sequential"] = round(served["speedup_vs_sequential"], 2)
    if lattices:
        out["lattices_ms"] = {name: {STRATEGY_NAMES[s]: round(row[STRATEGY_NAMES[s]]["ms"], 2) for s in range(4)}
                              for name, row in lattices.items()}
    return out


# ------------------------------------------------------------------------------------------
# Our arm
# ------------------------------------------------------------------------------------------

def main():
    args = parse_args()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    import torch.distributed as dist

    import back40computing_b200 as b

    rank, world, local = dist_info()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    g = make_graph(args.scale, args.edge_factor)
    sources = replica_sources(g, args.sources, rank)
    nsrc = len(sources)
    deg = g.degrees().astype(np.int64)
    strategies = [int(s) for s in args.strategies.split(",") if s.strip()]
    if HEADLINE not in strategies:
        strategies.insert(0, HEADLINE)

    stream = torch.cuda.Stream(device=dev)
    problem = b.CsrProblem(False).from_graph(g)
    problem.set_stream(stream.cuda_stream)

    def barrier():
        if world > 1:
            dist.barrier()

    # Oracle labels of the sources checked during warm-up (every source by
    # default), computed once on the host threads before any timing.
    nver = nsrc if args.verify < 0 else min(args.verify, nsrc)
    refs = None
    if nver:
        sys.path.insert(0, str(ROOT / "oracle"))
        from oracle import Oracle
        refs, _ = Oracle().bfs_many_labels(g, sources[:nver])
    results = {}
    checked = 0
    for strat in strategies:
        en = b.make_enactor(strat)
        en.set_stream(stream.cuda_stream)
        ft = en.GetFrontierType()
        E = np.zeros(nsrc, np.int64)
        V = np.zeros(nsrc, np.int64)
        # Warm-up steps; the first one also measures E and V per source and checks labels.
        for w in range(max(1, args.warmup)):
            for i, s in enumerate(sources):
                b.check(problem.ResetAsync(ft, 1.3))
                b.check(en.EnactSearchAsync(problem, int(s), 0, args.variant))
                if w == 0:
                    b.check(en.Sync())
                    lab = problem.labels()
                    vis = lab > -1
                    V[i] = int(vis.sum())
                    E[i] = int(deg[vis].sum())
                    if i < nver:
                        if not np.array_equal(lab, refs[i]):
                            bad = int(np.nonzero(lab != refs[i])[0][0])
                            raise SystemExit(f"bench: labels of strategy {strat} source {int(s)} differ from "
                                             f"the oracle at vertex {bad}")
                        checked += 1
            b.check(en.Sync())
        # Timed steps.
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps * nsrc)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps * nsrc)]
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local) if strat == HEADLINE else None
        if clocks:
            clocks.start()
        t_start.record(stream)
        k = 0
        for _ in range(args.steps):
            for s in sources:
                b.check(problem.ResetAsync(ft, 1.3))
                starts[k].record(stream)
                b.check(en.EnactSearchAsync(problem, int(s), 0, args.variant))
                ends[k].record(stream)
                k += 1
        t_end.record(stream)
        b.check(en.Sync())
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks else None
        total_ms = t_start.elapsed_time(t_end)
        kern_ms = [a.elapsed_time(z) for a, z in zip(starts, ends)]
        total_ms, edges_all = reduce_replicas(total_ms, float(E.sum()) * args.steps, world, dev)
        bytes_alg = 4.0 * E + 20.0 * V
        results[strat] = {
            "gteps": edges_all / (total_ms / 1e3) / 1e9,
            "ms_per_step": total_ms / args.steps,
            "kernel_ms_mean": float(np.mean(kern_ms)),
            "kernel_ms_median": float(np.median(kern_ms)),
            "alg_bytes_per_search": float(bytes_alg.mean()),
            "alg_gbs": float(bytes_alg.sum() * args.steps / (np.sum(kern_ms) / 1e3) / 1e9),
            "edges_visited_mean": float(E.mean()),
            "vertices_visited_mean": float(V.mean()),
            "verified_sources": min(nver, nsrc),
            # per search: Reset's initialisation kernel, the init kernel, the fused kernel
            "launches": 3 * args.steps * nsrc,
            "clocks": clk,
        }
        del en

    del refs

    # End-to-end through the public API with host buffers.
    e2e = None
    if not args.no_e2e:
        row_p = torch.from_numpy(g.row_offsets).pin_memory()
        col_p = torch.from_numpy(g.column_indices).pin_memory()
        E = np.zeros(nsrc, np.int64)
        # Two CsrProblems, each with its own enactor on its own stream, as a
        # caller that receives a stream of CSR uploads double-buffers them:
        # step k uploads into problem k % 2 while the other problem's searches
        # and label copies of step k - 1 are still running.
        streams2 = [stream, torch.cuda.Stream(device=dev)]
        probs, ens, outs = [], [], []
        for k in range(2):
            pr = b.CsrProblem(False)
            pr.set_stream(streams2[k].cuda_stream)
            en_k = b.make_enactor(HEADLINE)
            en_k.set_stream(streams2[k].cuda_stream)
            probs.append(pr)
            ens.append(en_k)
            outs.append([torch.empty(g.nodes, dtype=torch.int32).pin_memory() for _ in range(2)])
        ft = ens[0].GetFrontierType()

        def e2e_step(k, record, pipelined):
            prob, en = probs[k & 1], ens[k & 1]
            b.check(prob.FromHostProblem(False, g.nodes, g.edges, col_p.numpy(), row_p.numpy(), 1))
            for i, s in enumerate(sources):
                out = outs[k & 1][i & 1].numpy()
                if pipelined:  # two label buffers: the copy of search i overlaps search i + 1
                    b.check(prob.ResetAsync(ft, 1.3))
                    b.check(en.EnactSearchAsync(prob, int(s)))
                    b.check(prob.ExtractResultsAsync(out))
                else:
                    b.check(prob.Reset(ft, 1.3))
                    b.check(en.EnactSearch(prob, int(s)))
                    b.check(prob.ExtractResults(out))
                if record:
                    b.check(en.Sync())
                    b.check(prob.Sync())
                    E[i] = int(deg[out > -1].sum())

        def e2e_sync_all():
            for k in range(2):
                b.check(ens[k].Sync())
                b.check(probs[k].Sync())

        def e2e_time(pipelined):
            for pr in probs:
                pr.set_label_buffers(2 if pipelined else 1)
            for k in range(2 if pipelined else 1):
                e2e_step(k, True, pipelined)
            e2e_sync_all()
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for k in range(args.steps):
                # pipelined: alternate the two problems; synchronous: one problem
                e2e_step(k if pipelined else 0, False, pipelined)
            e2e_sync_all()
            torch.cuda.synchronize()
            return reduce_replicas(time.perf_counter() - t0, float(E.sum()) * args.steps, world, dev)

        secs_sync, edges_sync = e2e_time(False)
        secs, e2e_edges = e2e_time(True)
        e2e = {"value": e2e_edges / secs / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": int(4 * (g.nodes + 1) + 4 * g.edges),
               "d2h_bytes_per_step": int(4 * g.nodes * nsrc),
               "ms_per_step": secs / args.steps * 1e3,
               "step": "FromHostProblem (CSR from pinned host memory) + 64 x (ResetAsync, EnactSearchAsync, "
                       "ExtractResultsAsync to pinned host memory) with two label buffers; steps alternate two "
                       "CsrProblems, each with its own enactor and stream, so a step's upload overlaps the "
                       "previous step's searches and label copies; wall clock over all steps, then Sync",
               "synchronous_api": {"value": edges_sync / secs_sync / 1e9, "unit": UNIT,
                                   "ms_per_step": secs_sync / args.steps * 1e3,
                                   "step": "one CsrProblem, the synchronous FromHostProblem, Reset, EnactSearch, "
                                           "ExtractResults and one label buffer"}}
        for pr in probs:
            pr.close()
        del ens

    # Batched and served legs (one GPU; replicas add nothing to their comparison).
    batched = served = None
    if world == 1 and not args.no_batched:
        batched = batched_leg(b, torch, stream, args)
    if world == 1 and not args.no_served:
        served = served_leg(b, torch, stream, args, g)
    lattices = None
    if world == 1 and not args.no_lattices:
        lattices = lattice_leg(b, torch, stream, args)

    # CPU baseline: the reference's CPU BFS on a bounded sample, rank 0 at N=1.
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = np.take(sources, range(max(8, threads)), mode="wrap")
        e, dt, kind = run_cpu(g, sample, threads)
        cpu = {"value": e / dt / 1e9, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{len(sample)} of the 64 sources, one search per host thread, wall {dt:.2f} s"}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    head = results[HEADLINE]
    for st, r in results.items():
        # DRAM bytes of one launch (ncu, this workload) over the mean launch time.
        tr = measured_traffic(args.scale, st)
        r["dram_bytes_per_launch"] = tr
        r["dram_frac"] = None if tr is None else tr / (r["kernel_ms_mean"] / 1e3) / 1e9 / peak
        r["alg_frac"] = r["alg_gbs"] / peak
    traffic = head["dram_bytes_per_launch"]
    line = {
        "metric": METRIC, "value": head["gteps"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded R-MAT, 64 sources)",
        "config": bench_config(args, g.nodes, g.edges, nsrc, world),
        "summary": summary_block(e2e, batched, served, lattices, results),
        "headline": f"strategy {STRATEGY_NAMES[HEADLINE]} "
                    f"{'fused, direction-optimizing (alpha 14, beta 24)' if args.variant == 1 else 'iterative'}",
        "roofline": {"bound": "hbm", "achieved": head["alg_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": head["alg_gbs"] / peak, "traffic": traffic, "peak_source": peak_kind,
                     "dram_frac": head["dram_frac"],
                     "alg_bytes_per_launch": head["alg_bytes_per_search"],
                     "kernel_ms_mean": head["kernel_ms_mean"],
                     "note": "achieved = (4E + 20V) per search / fused-kernel time (of measured peak); traffic = "
                             "ncu DRAM bytes of one launch of the fused kernel on this workload; dram_frac = "
                             "traffic / mean kernel time / peak. The direction-optimizing search reads far fewer "
                             "bytes than 4E + 20V (bottom-up levels stop at the first parent)"},
        "verified": f"{checked} searches (every strategy x {min(nver, nsrc)} sources) bit-exact against the oracle "
                    f"during warm-up",
        "strategies": {STRATEGY_NAMES[s]: {k: v for k, v in r.items() if k != "clocks"} for s, r in results.items()},
        "gpu_launches": head["launches"],
        "clocks": head["clocks"],
        "e2e": e2e,
        "cpu_baseline": cpu,
        "batched": batched,
        "served": served,
        "lattices": lattices,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
