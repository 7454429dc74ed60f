"""Benchmark of the B200 BFS on the R-MAT scale-22 workload.

Workload (default): R-MAT scale 22, edge factor 16, a/b/c/d = .57/.19/.19/.05,
self-loops removed, duplicates kept, symmetrized (~134M int32 CSR entries);
64 sources drawn with seed 2 among vertices of degree > 0.  Synthetic, seeded.

A step is one BFS from each of the 64 sources (Reset + EnactSearch each).  The
headline strategy is expand-contract (fused persistent kernel); contract-expand
and two-phase are timed the same way and reported under "strategies".

  value   GTEPS = sum of edges_visited over the step's searches / device time,
          CSR resident in HBM, CUDA events on the enactor's stream.
  e2e     same metric through the public API with host buffers: every step
          uploads the CSR from pinned host memory (FromHostProblem), runs the 64
          searches and copies each label array back to pinned host memory.
  roofline  algorithmic bytes per search, 4E + 20V (column indices read once,
          a row-offset pair, a label write, a frontier write and read per
          visited vertex) / the fused kernel's average duration, against the
          measured HBM copy bandwidth.

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
STRATEGY_NAMES = {0: "expand_contract", 1: "contract_expand", 2: "two_phase"}
HEADLINE = 0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--strategies", default="0,1,2")
    ap.add_argument("--variant", type=int, default=1, help="1 fused, 2 iterative (graph-driven)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--verify", type=int, default=2, help="sources checked against the oracle")
    ap.add_argument("--sources", type=int, default=NUM_SOURCES, help="sources per step (64 for the bench line)")
    return ap.parse_args()


def dist_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def make_graph(scale, ef):
    from back40computing_b200 import graphs
    return graphs.rmat(scale, ef, 0.57, 0.19, 0.19, seed=1, undirected=True)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_traffic(scale):
    """DRAM bytes per launch of the headline kernel from the committed ncu
    summary (profiles/ec_fused_rmat21_full.md), scaled there to scale 22."""
    prof = ROOT / "profiles" / "ec_fused_rmat21_full.md"
    if scale != 22 or not prof.exists():
        return None
    for line in prof.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch_rmat22:"):
            return float(line.split(":", 1)[1])
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms in the background."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


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
    rank, world, _ = dist_info()
    if rank != 0:
        return
    g = make_graph(args.scale, args.edge_factor)
    sources = g.sample_sources(NUM_SOURCES, 2)
    threads = os.cpu_count() or 1
    per_step = max(8, threads)
    idx = 0
    for _ in range(args.warmup):
        sel = np.take(sources, range(idx, idx + per_step), mode="wrap")
        idx += per_step
        run_cpu(g, sel, threads)
    edges, secs = 0, 0.0
    kind = "port"
    for _ in range(args.steps):
        sel = np.take(sources, range(idx, idx + per_step), mode="wrap")
        idx += per_step
        e, dt, kind = run_cpu(g, sel, threads)
        edges += e
        secs += dt
    gteps = edges / secs / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": gteps, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded R-MAT)",
        "config": {"workload": f"rmat-s{args.scale}-ef{args.edge_factor} BFS, {per_step} of 64 sources per step",
                   "nodes": g.nodes, "edges": g.edges},
        "cpu_baseline": {"value": gteps, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{per_step} sources per step x {args.steps} steps, one search per host thread"},
        "e2e": {"value": gteps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


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
    sources = g.sample_sources(args.sources, 2 + 1000 * rank)
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

    results = {}
    verified = []
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
                    if i < args.verify:
                        verified.append((strat, int(s), lab))
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
        if world > 1:
            t = torch.tensor([total_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        edges_step = float(E.sum())
        bytes_alg = 4.0 * E + 20.0 * V
        results[strat] = {
            "gteps": edges_step * args.steps * world / (total_ms / 1e3) / 1e9,
            "ms_per_step": total_ms / args.steps,
            "kernel_ms_mean": float(np.mean(kern_ms)),
            "kernel_ms_median": float(np.median(kern_ms)),
            "alg_bytes_per_search": float(bytes_alg.mean()),
            "alg_gbs": float(bytes_alg.sum() * args.steps / (np.sum(kern_ms) / 1e3) / 1e9),
            "edges_visited_mean": float(E.mean()),
            "vertices_visited_mean": float(V.mean()),
            "launches": 2 * args.steps * nsrc,
            "clocks": clk,
        }
        del en

    # Labels of the warm-up runs checked bit-exact against the oracle.
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Oracle
    orc = Oracle()
    ref_cache = {}
    for strat, s, lab in verified:
        if s not in ref_cache:
            ref_cache[s] = orc.bfs(g, s)[0]
        if orc.first_mismatch(lab, ref_cache[s]) != -1:
            raise SystemExit(f"bench: labels of strategy {strat} source {s} differ from the oracle")

    # End-to-end through the public API with host buffers.
    e2e = None
    if not args.no_e2e:
        row_p = torch.from_numpy(g.row_offsets).pin_memory()
        col_p = torch.from_numpy(g.column_indices).pin_memory()
        outs = [torch.empty(g.nodes, dtype=torch.int32).pin_memory() for _ in range(2)]
        en = b.make_enactor(HEADLINE)
        en.set_stream(stream.cuda_stream)
        ft = en.GetFrontierType()
        E = np.zeros(nsrc, np.int64)

        def e2e_step(record):
            prob = b.CsrProblem(False)
            prob.set_stream(stream.cuda_stream)
            b.check(prob.FromHostProblem(False, g.nodes, g.edges, col_p.numpy(), row_p.numpy(), 1))
            for i, s in enumerate(sources):
                b.check(prob.Reset(ft, 1.3))
                b.check(en.EnactSearch(prob, int(s)))
                out = outs[i & 1].numpy()
                b.check(prob.ExtractResults(out))
                if record:
                    E[i] = int(deg[out > -1].sum())
            prob.close()

        e2e_step(True)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step(False)
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([secs], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            secs = float(t.item())
        e2e = {"value": float(E.sum()) * args.steps * world / secs / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": int(4 * (g.nodes + 1) + 4 * g.edges + 4 * nsrc),
               "d2h_bytes_per_step": int(4 * g.nodes * nsrc),
               "ms_per_step": secs / args.steps * 1e3}
        del en

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
    traffic = measured_traffic(args.scale)
    line = {
        "metric": METRIC, "value": head["gteps"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded R-MAT, 64 sources)",
        "config": {"workload": f"BFS rmat-s{args.scale}-ef{args.edge_factor} (a=.57 b=.19 c=.19), "
                               f"{nsrc} sources/step, strategy {STRATEGY_NAMES[HEADLINE]} "
                               f"{'fused' if args.variant == 1 else 'iterative'}",
                   "nodes": g.nodes, "edges": g.edges, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (column indices %.0f MB)" % (4 * g.edges / 1e6)},
        "roofline": {"bound": "hbm", "achieved": head["alg_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": head["alg_gbs"] / peak, "traffic": traffic, "peak_source": peak_kind,
                     "alg_bytes_per_launch": head["alg_bytes_per_search"],
                     "kernel_ms_mean": head["kernel_ms_mean"]},
        "strategies": {STRATEGY_NAMES[s]: {k: v for k, v in r.items() if k != "clocks"} for s, r in results.items()},
        "gpu_launches": head["launches"],
        "clocks": head["clocks"],
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
