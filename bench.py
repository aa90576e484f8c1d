#!/usr/bin/env python3
"""Loopy belief-propagation throughput on one B200 (or N, one process each).

Workload (default): loopy BP on a 16,777,216-node, 67,108,864-edge graph with
power-law out-degree (exponent 2.5, min 1, mean 4), uniform destinations,
2 states, row-normalised U(0,1) joint tables, Dirichlet(1) priors, 10%
one-hot evidence, synchronous flooding schedule, 100 fixed iterations
(tolerance 0), seed 1.  One step = one BP solve as the reference times it
(c_benchmark/main.c:277-281): reset beliefs to the priors,
init_previous_edge, loopy_propagate_until.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bp|reference]

value  edge-msg updates/s over the whole job (E * iterations * N / max-rank time),
       graph resident in HBM.
e2e    the same metric through the public C-ABI with host (pinned) buffers:
       every step uploads the graph (edges, tables, priors), builds the
       destination-sorted layout on the GPU, runs, and reads the beliefs back;
       the steps are pipelined as a serving loop runs them (step k+1's upload
       and build on a second stream and host thread, and step k-1's read-back
       on a third host thread, during step k's solve),
       timed by wall clock from the first upload to the last read; the
       median of three such runs.  The loop reserves its device memory once
       at start-up (bp_reserve_cached_memory).
Multi-GPU: independent replicas, one per rank (weak scaling), no collective
on the data path; the timing is the max over ranks.  --shard splits the one
graph over the ranks by destination-node ranges instead.
On one GPU the headline line also carries `other_configs`: the lines of the
other workloads (random10k, tree, batched, unrolled, unrolled_batch), each
run in a child process after the headline (--configs none skips them).
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edge-msg updates/s"
UNIT = "edge-msg updates/s"
FALLBACK_HBM_GBS = 6650.0


def max_over_ranks(value, dist, device="cuda"):
    """The largest `value` over all ranks (every rank calls this at the same
    point); `value` itself when running alone."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["bp", "reference"], default="bp")
    ap.add_argument("--iterations", type=int, default=100)
    ap.add_argument("--nodes", type=int, default=1 << 24)
    ap.add_argument("--edges", type=int, default=1 << 26)
    # steps of a timed serving-loop run: the first build is not overlapped,
    # so fewer steps weigh the pipeline fill more (6 steps: 94.5 ms per step,
    # 12 steps: 91.8 ms on the 16.8M-node graph)
    ap.add_argument("--e2e-steps", type=int, default=12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--batch-delta", choices=["serial", "f64"], default="f64",
                    help="batched workload's stopping rule: the reference's serial fp32 delta (decided by "
                         "bounds) or a deterministic fp64 sum")
    ap.add_argument("--workload", choices=["power_law", "random10k", "batched", "tree", "unrolled",
                                           "unrolled_batch"],
                    default="power_law",
                    help="power_law: the headline loopy workload; batched: 4096 independent networks; "
                         "tree: tree BP on a 2M-node random recursive tree")
    ap.add_argument("--tree-nodes", type=int, default=2_000_000)
    ap.add_argument("--shard", action="store_true",
                    help="split the one graph over the ranks by destination-node ranges (strong scaling: send "
                         "buffers all-gathered every iteration) instead of one replica per rank")
    ap.add_argument("--reorder", type=int, default=1,
                    help="1: renumber nodes by out-degree inside the engine (results unchanged)")
    ap.add_argument("--networks", type=int, default=4096)
    ap.add_argument("--grids", type=int, default=256,
                    help="unrolled_batch: the first N of the 256 grids (smaller profiling cases)")
    ap.add_argument("--solo-sample", type=int, default=256,
                    help="batched: networks solved one launch sequence each, for the comparison")
    ap.add_argument("--configs", choices=["all", "none"], default="all",
                    help="headline run on one GPU: also run every other workload (one child process each, "
                         "after the headline's timed region) and attach their results under other_configs")
    return ap.parse_args()


OTHER_WORKLOADS = ("random10k", "tree", "batched", "unrolled", "unrolled_batch")
OTHER_KEYS = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "higher_is_better", "config", "clocks",
              "max_abs_err_vs_oracle", "max_abs_err_vs_fp64", "fp64_iterations", "iterations", "roofline",
              "cpu_baseline", "forward_ms", "fwd_bwd_over_fwd", "plain_forward_ms", "networks_per_s_fwd_bwd",
              "gpu_launches")


def run_other_configs(a):
    """Every other workload, each as `bench.py --workload W` in a child
    process on the same GPU (its own clock record), run after the headline's
    timed region; returns {workload: the fields of its JSON line} (or the
    error a workload ended with, which does not fail the headline)."""
    out = {}
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE")}
    for w in OTHER_WORKLOADS:
        cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--workload", w, "--warmup", str(max(a.warmup, 3))]
        t0 = time.time()
        try:
            r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
            lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
            if r.returncode != 0 or not lines:
                out[w] = {"error": f"exit {r.returncode}: " + (r.stderr or r.stdout)[-300:]}
            else:
                d = json.loads(lines[-1])
                out[w] = {k: d[k] for k in OTHER_KEYS if k in d}
        except subprocess.TimeoutExpired:
            out[w] = {"error": "did not finish in 900 s"}
        out[w]["wall_s"] = round(time.time() - t0, 1)
    return out


def workload_name(a):
    return (f"loopy BP, power-law out-degree graph: {a.nodes:,} nodes, {a.edges:,} edges, 2 states, "
            f"{a.iterations} fixed iterations, seed 1")


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(name, key="traffic_bytes_per_launch"):
    """DRAM bytes per launch (or per iteration, with that key) of the
    flooding kernels from the committed ncu summary (profiles/<name>), or
    None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + ":"):
            return float(line.split(":", 1)[1])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once the sampler reports (nvidia-smi
            # takes a moment to start), so short regions still get samples
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _restatement(openmp=True):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O, O.Restatement(openmp=openmp)


def fp64_error_loopy(net, tol, max_it, gpu_beliefs, gpu_iterations, what):
    """Accuracy of a GPU loopy run (the checker's leg, after the timed region):
    max |b_gpu - b| against the oracle's fp32 run of the same schedule (the
    reference's arithmetic; 0 means bit-identical) and against the oracle's
    fp64 run of the same schedule, with each run's returned iteration count.
    The oracle's OpenMP build runs the node loops on all host cores."""
    O, R = _restatement()
    og = O.OracleGraph(net)
    S = int(net.s_max)
    f32 = R.loopy(og, tol, max_it)
    f64 = R.loopy(og, tol, max_it, dtype=np.float64)
    b = np.asarray(gpu_beliefs, np.float64)[:, :S]
    return {"max_abs_err_vs_oracle": float(np.abs(b - f32["beliefs"][:, :S]).max()) if net.V else 0.0,
            "max_abs_err_vs_fp64": float(np.abs(b - f64["beliefs"][:, :S]).max()) if net.V else 0.0,
            "iterations": int(gpu_iterations), "oracle_iterations": int(f32["ret"]),
            "fp64_iterations": int(f64["ret"]), "fp64_delta": float(f64["delta"]), "sample": what}


def fp64_error_curve(net, graph, checkpoints=(1, 2, 5, 10, 20, 50, 100)):
    """How far the fp32 schedule (the reference's arithmetic, which the GPU
    reproduces bit for bit) drifts from the same schedule in fp64, iteration
    by iteration, tolerance 0: the GPU graph `graph` and the oracle's fp32 and
    fp64 runs are continued from checkpoint to checkpoint (each continuation
    recomputes the send buffers from the beliefs and latest messages, as the
    next iteration would).  The reference's update multiplies each belief
    into itself every iteration, so beliefs saturate towards 0/1 and a node
    whose fp32 and fp64 runs tip opposite ways shows an error near 1."""
    O, R = _restatement()
    og = O.OracleGraph(net)
    S = int(net.s_max)
    graph.set_beliefs(net.beliefs)
    graph.latest_slot = 1
    graph.init_messages()
    st = {}
    done = 0
    out = []
    for k in checkpoints:
        graph.loopy(0.0, k - done, delta="f64")
        b_gpu = graph.beliefs().astype(np.float64)[:, :S]
        row = {"iterations": k}
        for dt, name in ((np.float32, "oracle"), (np.float64, "fp64")):
            prev = st.get(name)
            if prev is None:
                r = R.loopy(og, 0.0, k, dtype=dt)
            else:
                r = R.loopy(og, 0.0, k - done, dtype=dt, init=False, beliefs=prev["beliefs"],
                            msgs=(prev["latest"], prev["older"]))
            st[name] = r
            row[f"max_abs_err_vs_{name}"] = float(np.abs(b_gpu - r["beliefs"][:, :S]).max())
        ref64 = st["fp64"]["beliefs"][:, :S]
        row["argmax_differs_vs_fp64"] = float(np.mean(b_gpu.argmax(1) != ref64.argmax(1)))
        row["nodes_off_by_1e-5_vs_fp64"] = float(np.mean(np.abs(b_gpu - ref64).max(1) > 1e-5))
        out.append(row)
        done = k
    return out


def flood_bytes_per_iteration(V, E, S):
    """Compulsory HBM bytes of one fused flooding iteration (loopy.cu header)."""
    return E * (4 * S * S + 4 + 4 * S * 3) + V * (4 + 4 * S * 3)


# ---------------------------------------------------------------- CPU side
def reference_sample(iterations=None, target_s=10.0):
    """The reference's own graph.c (OpenMP build, all host cores) on a bounded
    sample of the same workload: 1,048,576 nodes / 4,194,304 edges of the same
    generator, fixed iterations.  Returns the baseline dict or None."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import belief_network_wrapper as W
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    kind = "reference"
    if O.reference_available(openmp=True):
        ref = O.Reference(openmp=True)
    else:
        kind, cores = "port", 1
        ref = None
    net = W.bp.synth.power_law_loopy(1 << 20, 1 << 22, 2, 0.10, seed=1)

    def run(iters):
        if ref is not None:
            g = ref.build_graph(net)
            # graph.c prints "No Convergence" on stdout when the fixed
            # iteration count runs out; keep stdout for the JSON line
            sys.stdout.flush()
            saved = os.dup(1)
            devnull = os.open(os.devnull, os.O_WRONLY)
            os.dup2(devnull, 1)
            try:
                t0 = time.perf_counter()
                ref.lib.init_previous_edge(g)
                ref.lib.loopy_propagate_until(g, 0.0, iters)
                dt = time.perf_counter() - t0
            finally:
                os.dup2(saved, 1)
                os.close(saved)
                os.close(devnull)
            ref.lib.graph_destroy(g)
            return dt
        R = O.Restatement()
        og = O.OracleGraph(net)
        t0 = time.perf_counter()
        R.loopy(og, 0.0, iters)
        return time.perf_counter() - t0

    if iterations is None:
        probe = run(2)
        iterations = int(max(2, min(200, target_s / max(probe / 2, 1e-6))))
    dt = run(iterations)
    return {"value": net.E * iterations / dt, "unit": UNIT, "cores": int(os.environ.get("OMP_NUM_THREADS", cores))
            if kind == "reference" else 1, "kind": kind,
            "sample": f"{net.V:,} nodes / {net.E:,} edges of the same generator, {iterations} fixed iterations, "
                      f"init_previous_edge + loopy_propagate_until timed ({dt:.2f} s)",
            "seconds": dt, "iterations": iterations}


def power_law_accuracy(a, handle):
    """The GPU's beliefs after the workload's fixed iterations on the
    1,048,576-node sample of the same generator (the CPU baseline's sample,
    small enough for the fp64 oracle), same code path as the timed run."""
    import belief_network_wrapper as W
    from belief_propagation_b200.engine import BPGraph
    net = W.bp.synth.power_law_loopy(1 << 20, 1 << 22, 2, 0.10, seed=1)
    g = BPGraph(net.V, net.src, net.dst, net.joint, uniform_states=2, stream=handle, reorder=bool(a.reorder))
    try:
        g.set_beliefs(net.beliefs)
        g.latest_slot = 1
        g.init_messages()
        r = g.loopy(0.0, a.iterations, delta="f64")
        b = g.beliefs()
        out = fp64_error_loopy(net, 0.0, a.iterations, b, r["iterations"],
                               f"{net.V:,} nodes / {net.E:,} edges of the same generator, {a.iterations} fixed "
                               "iterations, same code path")
        out["by_iteration"] = fp64_error_curve(net, g, tuple(k for k in (1, 2, 5, 10, 20, 50, 100)
                                                             if k <= a.iterations))
    finally:
        g.close()
    return out


def run_sharded(a, rank, world, net, gen_s, dist, barrier, local):
    """The headline graph split over the ranks by destination-node ranges
    (belief_propagation_b200.sharded): each rank holds its nodes' in-edges and
    runs bp_flood_range on them; the send buffers are all-gathered over NCCL
    and the deltas summed in rank order after every iteration.  value = the
    whole job's edge-msg updates/s (strong scaling: the graph is fixed)."""
    import torch
    from belief_propagation_b200.sharded import LocalComm, RangeEngine, TorchComm, node_ranges, sharded_loopy
    ranges, chunk = node_ranges(net.V, world)
    eng = RangeEngine(net, *ranges[rank], chunk, world)
    comm = TorchComm(dist, rank, chunk) if dist is not None else LocalComm(chunk)
    prior = torch.from_numpy(net.beliefs).cuda()

    def step():
        return sharded_loopy([eng], comm, prior, 0.0, a.iterations)

    for _ in range(a.warmup):
        step()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record()
    for _ in range(a.steps):
        r = step()
    ev1.record()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist) / a.steps
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": float(net.E) * a.iterations / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(a), "nodes": net.V, "edges": net.E, "states": 2,
                       "iterations": a.iterations, "parallelism": f"destination-range split x{world}",
                       "node_order": "caller ids", "generator_s": round(gen_s, 1),
                       "exchange": "send buffers all-gathered (NCCL) and deltas summed in rank order, every "
                                   "iteration"},
            "executed": r["executed"], "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_arm(a, rank, world):
    if rank != 0:
        return 0
    iters = None
    steps = []
    for i in range(a.warmup + a.steps):
        r = reference_sample(iterations=iters, target_s=3.0)
        iters = r["iterations"]
        if i >= a.warmup:
            steps.append(r)
    tot = sum(s["seconds"] for s in steps)
    value = sum(s["value"] * s["seconds"] for s in steps) / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * tot / len(steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": workload_name(a), "arm": "reference CPU (OpenMP graph.c)",
                                            "step": steps[0]["sample"]},
            "cpu_baseline": {k: steps[0][k] for k in ("kind", "cores", "sample")} | {"value": value, "unit": UNIT},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU side
def run_batched(a, rank, world):
    """Batched loopy BP: independent random networks (node counts
    log-uniform in [32, 4096], edges U(2,6) x nodes, states uniform in
    {2,3,4,8} per network, Dirichlet(1) priors, row-normalised U(0,1) tables,
    10% evidence), tolerance 1e-4 per network with early exit, at most 200
    iterations, seed 2.  One step = the whole batch solved from its priors
    (init_previous_edge + loopy_propagate_until per network) in one CUDA
    graph launch.  Compared with solving a sample of the same networks one
    at a time through bp_loopy (one launch sequence per network)."""
    import torch
    import belief_network_wrapper as W
    from belief_propagation_b200.engine import BPBatch, BPGraph

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    t0 = time.time()
    nets = W.bp.synth.batch_of_networks(count=a.networks, seed=2)
    gen_s = time.time() - t0
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    handle = stream.cuda_stream
    b = BPBatch(nets, stream=handle)
    prior = torch.from_numpy(b.pack_beliefs()).cuda()
    b.set_beliefs(prior)
    tuned = b.autotune(tol=1e-4, max_iterations=200, delta=a.batch_delta)
    groups = b.groups()

    def step():
        b.set_beliefs(prior)
        return b.loopy(tol=1e-4, max_iterations=200, delta=a.batch_delta)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        r = step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / a.steps
    ms = max_over_ranks(ms, dist)
    res = b.results()
    flat = b.beliefs()
    edges = sum(n.E for n in nets)
    updates = float(res["executed"].astype(np.float64) @ np.array([n.E for n in nets], np.float64))

    # one network at a time through bp_loopy: graphs resident, each solve its
    # own launch sequence and host synchronisation
    rng = np.random.default_rng(0)
    sample = sorted(rng.choice(len(nets), size=min(a.solo_sample, len(nets)), replace=False).tolist())
    graphs = [BPGraph.from_network(nets[k], stream=handle) for k in sample]
    priors = [torch.from_numpy(nets[k].beliefs).cuda() for k in sample]

    def solo_all():
        for g, p in zip(graphs, priors):
            g.set_beliefs(p)
            g.latest_slot = 1
            g.init_messages()
            g.loopy(1e-4, 200, delta=a.batch_delta)

    solo_all()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    solo_all()
    torch.cuda.synchronize()
    solo_s = time.perf_counter() - t1
    for g in graphs:
        g.close()
    solo_nets_s = len(sample) / solo_s
    b.close()
    accuracy = None
    if rank == 0:
        # the oracle's fp32 and fp64 runs of 64 sampled networks, each alone
        try:
            acc_sample = sorted(np.random.default_rng(1).choice(len(nets), size=min(64, len(nets)),
                                                                replace=False).tolist())
            errs = []
            for k in acc_sample:
                n = nets[k]
                S = n.uniform_states
                o = int(b.belief_off[k])
                bk = flat[o:o + n.V * S].reshape(n.V, S)
                errs.append(fp64_error_loopy(n, 1e-4, 200, bk, int(res["iterations"][k]), ""))
            accuracy = {"max_abs_err_vs_oracle": max(e["max_abs_err_vs_oracle"] for e in errs),
                        "max_abs_err_vs_fp64": max(e["max_abs_err_vs_fp64"] for e in errs),
                        "fp64_iterations_equal": sum(e["fp64_iterations"] == e["iterations"] for e in errs),
                        "oracle_iterations_equal": sum(e["oracle_iterations"] == e["iterations"] for e in errs),
                        "sample": f"{len(acc_sample)} networks of the batch (seeded choice), each run alone by "
                                  "the oracle in fp32 (the reference's serial stopping rule) and in fp64 (its own "
                                  "stopping rule), tol 1e-4, max 200"}
        except Exception as ex:  # reported, not fatal
            accuracy = {"error": str(ex)[:200]}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    value = a.networks * world / (ms / 1e3)
    # algorithmic bytes: each network's fused-iteration bytes times the
    # iterations it ran, plus its prologue (messages from the priors, then Q)
    algo = 0.0
    for n, it in zip(nets, res["executed"].tolist()):
        S = int(n.s_max)
        algo += it * flood_bytes_per_iteration(n.V, n.E, S)
        algo += n.E * (4 * S * S + 4 + 4 * S + 4 * S) + n.V * (4 + 4 * S + 4 * S)
    peak, peak_src = measured_hbm_peak()
    achieved = algo / (ms / 1e3) / 1e9
    # no HBM roofline: a block iterates one network to convergence and the
    # network's arrays (<= ~1 MB) stay in L2 across its iterations, so these
    # bytes are mostly L2 traffic, and no measured L2 peak is at hand
    roofline = {"bound": "l2 / latency", "achieved": achieved, "peak": None, "unit": "GB/s", "frac": None,
                "traffic": None, "kernel": "k_batch_solve", "peak_source": None,
                "algorithmic_bytes_per_step": algo,
                "note": "algorithmic bytes per second, mostly served from L2; not a fraction of the HBM peak"}
    line = {"metric": "batched nets/s", "value": value, "unit": "networks/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{a.networks} independent networks, V log-uniform [32,4096], E U(2,6)xV, "
                                   "S in {2,3,4,8}, tol 1e-4 per network, max 200 iterations, seed 2",
                       "delta": a.batch_delta + (" (the reference's serial fp32 stopping rule, decided by bounds)"
                                                 if a.batch_delta == "serial" else " (deterministic fp64 sum)"),
                       "nodes": int(sum(n.V for n in nets)), "edges": int(edges), "block_threads": tuned, "groups": groups,
                       "generator_s": round(gen_s, 1), "l2": "batch working set larger than L2"},
            "converged": int(r["converged"]), "max_iterations_run": int(r["max_executed"]),
            "edge_msg_updates_per_s": updates / (ms / 1e3),
            "per_network_launches": {"sample": len(sample), "networks_per_s": solo_nets_s,
                                     "speedup_of_batched": value / world / solo_nets_s},
            "roofline": roofline, "gpu_launches": len(tuned) * a.steps, "clocks": clk}
    if accuracy is not None:
        line.update({k: accuracy[k] for k in ("max_abs_err_vs_oracle", "max_abs_err_vs_fp64") if k in accuracy})
        line["accuracy"] = accuracy
    print(json.dumps(line), flush=True)
    return 0


def run_random10k(a, rank, world):
    """The reference-runnable workload: 10,000 nodes, 40,000 uniform random
    edges, 2 states, 10% evidence, tol 1e-3, max 100 iterations, seed 0.  One
    step = init_previous_edge + loopy_propagate_until from the priors with the
    reference's own serial fp32 delta stopping rule (decided from the f64 sum
    and the serial sum's rounding bound, the serial sum formed only where the
    bound straddles the tolerance; the same iteration count by construction),
    through the drop-in-equivalent device API.  The reference's graph.c runs
    the same full workload on one host core beside it."""
    import torch
    import belief_network_wrapper as W
    from belief_propagation_b200.engine import BPGraph
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    net = W.bp.synth.random_loopy(10_000, 40_000, 2, 0.10, seed=0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    g = BPGraph.from_network(net, stream=stream.cuda_stream)
    prior = torch.from_numpy(net.beliefs).cuda()

    def step(delta):
        g.set_beliefs(prior)
        g.latest_slot = 1
        g.init_messages()
        return g.loopy(1e-3, 100, delta=delta)

    res = {}
    # about 1.5 s of solves per mode, so the clock sampler sees the region
    reps = max(a.steps, 1000)
    clocks = ClockSampler(local)
    clocks.start()
    for delta in ("serial", "f64"):
        for _ in range(a.warmup):
            r = step(delta)
        ms = _time_cuda(lambda: step(delta), stream, reps)
        res[delta] = (ms, r["iterations"], r["executed"], r["serial_sums"], g.beliefs())
    clk = clocks.stop()
    b_gpu = res["serial"][4]
    curve = None
    if rank == 0:
        try:
            curve = fp64_error_curve(net, g)
        except Exception as ex:  # reported, not fatal
            curve = [{"error": str(ex)[:200]}]
    g.close()
    cpu = None
    if O.reference_available():
        ref = O.Reference()
        rg = ref.build_graph(net)
        t0 = time.perf_counter()
        ref.lib.init_previous_edge(rg)
        it_ref = ref.lib.loopy_propagate_until(rg, 1e-3, 100)
        cpu_s = time.perf_counter() - t0
        b_ref = np.zeros((net.V, 10), np.float32)
        ref.lib.refshim_get_beliefs(rg, b_ref)
        ref.lib.graph_destroy(rg)
        cpu = {"value": 1e3 * cpu_s, "unit": "ms per solve", "cores": 1, "kind": "reference",
               "sample": f"the full workload on the reference's graph.c (serial), returned {it_ref}; GPU beliefs "
                         f"bit-identical: {bool(np.array_equal(b_ref[:, :2], b_gpu))}"}
    accuracy = None
    if rank == 0:
        try:
            accuracy = fp64_error_loopy(net, 1e-3, 100, b_gpu, res["serial"][1],
                                        "the full workload, the reference's serial fp32 stopping rule")
            accuracy["by_iteration"] = curve
        except Exception as ex:  # reported, not fatal
            accuracy = {"error": str(ex)[:200]}
    if rank != 0:
        return 0
    ms, it, ex, sums, _ = res["serial"]
    line = {"metric": "loopy BP ms per solve (reference-runnable workload)", "value": ms, "unit": "ms",
            "n_gpus": 1, "steps": max(a.steps, 10), "warmup": a.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "replicas", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "10,000 nodes, 40,000 edges, 2 states, 10% evidence, tol 1e-3, max 100, seed 0",
                       "iterations_returned": it, "iterations_run": ex,
                       "serial_sums_formed": sums},
            "us_per_iteration": 1e3 * ms / max(ex, 1), "edge_msg_updates_per_s": 40_000 * ex / (ms / 1e3),
            "f64_delta_ms_per_solve": res["f64"][0], "cpu_baseline": cpu, "clocks": clk}
    if accuracy is not None:
        line.update({k: accuracy[k] for k in ("max_abs_err_vs_oracle", "max_abs_err_vs_fp64", "fp64_iterations")
                     if k in accuracy})
        line["accuracy"] = accuracy
    print(json.dumps(line), flush=True)
    return 0


def run_tree(a, rank, world):
    """Tree BP (c_benchmark/main.c:224-236) on a random recursive tree: parent
    of node i uniform in [0, i), both directions, states per node uniform in
    {2,3,4,8}, row-normalised U(0,1) tables, 5% evidence, seed 1.  One step =
    start pass, forward levels, reset, backward levels, marginalize, on the
    device; the O(V+E) level build is timed separately (the reference's is
    O(V^2)).  Checked bit for bit against the oracle's restatement at full
    size, which is also the CPU baseline (port, 1 core)."""
    import torch
    import belief_network_wrapper as W
    from belief_propagation_b200.engine import BPGraph
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    net = W.bp.synth.random_tree(a.tree_nodes, (2, 3, 4, 8), 0.05, seed=1)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    g = BPGraph.from_network(net, stream=stream.cuda_stream)
    t0 = time.perf_counter()
    lv, nl = g.build_levels()
    levels_s = time.perf_counter() - t0
    prior = torch.from_numpy(net.beliefs).cuda()

    def step():
        g.set_beliefs(prior)
        return g.tree()

    for _ in range(a.warmup):
        r = step()
    torch.cuda.synchronize()
    # at least ~2 s of trees, so the clock sampler sees the timed region
    t0 = time.perf_counter()
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    per = (time.perf_counter() - t0) / 3
    steps = max(a.steps, int(2.0 / max(per, 1e-4)))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    clocks.start()
    e0.record(stream)
    for _ in range(steps):
        r = step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / steps
    b_gpu = g.beliefs()
    g.close()
    cpu = None
    accuracy = None
    if rank == 0:
        R = O.Restatement()
        og = O.OracleGraph(net)
        t0 = time.perf_counter()
        ora = R.tree(og)
        cpu_s = time.perf_counter() - t0
        S = net.s_max
        same = bool(np.array_equal(b_gpu, ora["beliefs"][:, :S]))
        cpu = {"value": 1e3 * cpu_s, "unit": "ms per tree (levels + passes)", "cores": 1, "kind": "port",
               "sample": f"the full tree, oracle restatement (O(V+E) levels), bit-identical to the GPU: {same}"}
        o64 = R.tree(og, dtype=np.float64)
        bg = b_gpu.astype(np.float64)
        accuracy = {"max_abs_err_vs_oracle": float(np.abs(bg - ora["beliefs"][:, :S]).max()),
                    "max_abs_err_vs_fp64": float(np.abs(bg - o64["beliefs"][:, :S]).max()),
                    "sample": "the full tree; tree BP runs a fixed schedule (no iteration count)"}
    if rank != 0:
        return 0
    # algorithmic bytes of one tree: two passes over the edges (tables
    # S_src x S_dst, the source buffer and the message) and the nodes, plus
    # the marginalize pass
    ss = net.num_states[net.src].astype(np.float64)
    sd = net.num_states[net.dst].astype(np.float64)
    sv = net.num_states.astype(np.float64)
    per_pass = float((4 * ss * sd + 8 * ss).sum() + (12 * sv + 8).sum())
    algo = 2 * per_pass + float((4 * sv * 2 + 8).sum())
    peak, peak_src = measured_hbm_peak()
    achieved = algo / (ms / 1e3) / 1e9
    roofline = {"bound": "latency (levels and waves)", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "kernel": "k_tree_wave", "peak_source": peak_src,
                "algorithmic_bytes_per_tree": algo}
    line = {"metric": "tree BP ms per tree", "value": ms, "unit": "ms", "n_gpus": 1, "steps": steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "replicas",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"tree BP, random recursive tree, {net.V:,} nodes, {net.E:,} edges, "
                                   "states {2,3,4,8}, 5% evidence, seed 1",
                       "levels": nl, "waves": r["num_waves"], "level_build_s": levels_s},
            "nodes_per_s": net.V / (ms / 1e3), "roofline": roofline, "cpu_baseline": cpu,
            "gpu_launches": (r["num_waves"] + 5) * steps,
            "clocks": clk}
    if accuracy is not None:
        line.update({k: accuracy[k] for k in ("max_abs_err_vs_oracle", "max_abs_err_vs_fp64")})
        line["accuracy"] = accuracy
    print(json.dumps(line), flush=True)
    return 0


def ce_loss(log_beliefs, labels):
    """Cross-entropy of log-beliefs against integer labels, the mean over nodes
    (the value of torch's nll_loss with reduction='mean'): the library's fused
    loss head, one launch forward and one backward (a gather, a mean and the
    scatter of their gradient took eight generic kernels, 44 us per step)."""
    from belief_propagation_b200.unrolled import nll_loss
    return nll_loss(log_beliefs, labels)


def _time_cuda(fn, stream, reps):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def unrolled_fp64_error(eng, theta, Wp, labels, srcs, dsts, tabs, sides, S, T, batch):
    """fp32 engine against the pure-torch unrolled reference in fp64
    (autograd through every step): beliefs and both gradients of the
    cross-entropy.  The whole grid for the single-grid workload; for the
    batch, the first 8 grids through an engine of their own (the batch's
    gradient of the shared table sums over every grid)."""
    import torch
    from belief_propagation_b200.unrolled import UnrolledBP, torch_unrolled
    k = 8 if batch else 1
    Vs = int(sum(int(s) * int(s) for s in sides[:k]))
    src = np.concatenate(srcs[:k]).astype(np.uint32)
    dst = np.concatenate(dsts[:k]).astype(np.uint32)
    tab = np.concatenate(tabs[:k])
    sub_eng = UnrolledBP(Vs, src, dst, tab, S, T, checkpoint_every=5) if batch else eng
    th = theta.detach()[:Vs].clone().requires_grad_(True)
    W = Wp.detach().clone().requires_grad_(True)
    lab = labels[:Vs]
    lb = sub_eng(th, W)
    ce_loss(lb, lab).backward()
    th64 = th.detach().double().requires_grad_(True)
    W64 = W.detach().double().requires_grad_(True)
    lb64 = torch_unrolled(th64, W64, src, dst, tab, T)
    torch.nn.functional.nll_loss(lb64, lab).backward()
    out = {"max_abs_err_vs_fp64": float((lb.detach().double().exp() - lb64.detach().exp()).abs().max()),
           "grad_log_unary_max_rel_err_vs_fp64": float((th.grad.double() - th64.grad).abs().max()
                                                        / th64.grad.abs().max()),
           "grad_log_pair_max_rel_err_vs_fp64": float((W.grad.double() - W64.grad).abs().max()
                                                       / W64.grad.abs().max()),
           "sample": (f"the first {k} grids ({Vs:,} nodes), an engine of their own" if batch else "the whole grid")
           + "; pure-torch unrolled reference in fp64, autograd"}
    if batch:
        sub_eng.close()
    del lb64, th64, W64
    torch.cuda.empty_cache()
    return out


def run_unrolled(a, rank, world, batch):
    """Differentiable unrolled loopy BP.
    unrolled:       512x512 4-neighbour grid, 4 states, unary N(0,1), one shared
                    4x4 pairwise log-potential N(0,0.5), T=30, checkpoints every 5,
                    cross-entropy against uniform random labels, seed 3.
    unrolled_batch: 256 grids of side U[32,256], 8 states, same potentials,
                    T=20, one forward and one backward over the whole batch (its
                    disjoint union), then 50 SGD steps (lr 0.1) on the shared table,
                    seed 4.
    Reports forward ms, forward+backward ms and their ratio, next to the plain
    engine's forward (bp_loopy, T fixed iterations) on the same graph."""
    import torch
    import belief_network_wrapper as W
    from belief_propagation_b200.engine import BPGraph
    from belief_propagation_b200.unrolled import UnrolledBP

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    synth = W.bp.synth
    if batch:
        rng = np.random.default_rng(4)
        sides = rng.integers(32, 257, size=256)[: a.grids]
        S, T = 8, 20
    else:
        rng = np.random.default_rng(3)
        sides = np.array([512])
        S, T = 4, 30
    srcs, dsts, tabs, off = [], [], [], 0
    for side in sides:
        s_, d_, fwd = synth.grid_edges(int(side))
        srcs.append(s_.astype(np.int64) + off)
        dsts.append(d_.astype(np.int64) + off)
        tabs.append(np.where(fwd, 0, 0x80).astype(np.uint8))
        off += int(side) * int(side)
    V = off
    src = np.concatenate(srcs).astype(np.uint32)
    dst = np.concatenate(dsts).astype(np.uint32)
    tab = np.concatenate(tabs)
    E = len(src)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    theta = torch.tensor(rng.normal(0, 1, (V, S)), dtype=torch.float32, device="cuda", requires_grad=True)
    Wp = torch.tensor(rng.normal(0, 0.5, (1, S, S)), dtype=torch.float32, device="cuda", requires_grad=True)
    labels = torch.tensor(rng.integers(0, S, V), device="cuda")
    eng = UnrolledBP(V, src, dst, tab, S, T, checkpoint_every=5)

    def fwd():
        with torch.no_grad():
            return eng(theta, Wp)

    def fwd_bwd():
        theta.grad = None
        Wp.grad = None
        lb = eng(theta, Wp)
        loss = ce_loss(lb, labels)
        loss.backward()
        return loss

    for _ in range(a.warmup):
        fwd_bwd()
    # enough repetitions for about a second of forward+backward, so that the
    # clock sampler sees the timed region
    est = _time_cuda(fwd_bwd, stream, 3)
    reps = max(a.steps, 3, int(1000.0 / max(est, 1e-3)))
    clocks = ClockSampler(local)
    clocks.start()
    f_ms = _time_cuda(fwd, stream, reps)
    fb_ms = _time_cuda(fwd_bwd, stream, reps)
    clk = clocks.stop()
    # the plain engine's forward on the same graph and tables, T iterations
    E_tab = np.exp(Wp.detach().cpu().numpy()[0])
    joint = np.where((tab & 0x80)[:, None, None] != 0, E_tab.T[None], E_tab[None]).astype(np.float32)
    prior = torch.softmax(theta.detach(), 1)
    g = BPGraph(V, src, dst, joint, uniform_states=S, stream=stream.cuda_stream)

    def plain():
        g.set_beliefs(prior)
        g.latest_slot = 1
        g.init_messages()
        g.loopy(0.0, T, delta="f64")

    plain()
    p_ms = _time_cuda(plain, stream, reps)
    b_plain = g.beliefs()
    g.close()
    b_unrolled = np.exp(fwd().cpu().numpy())
    max_diff = float(np.abs(b_plain - b_unrolled).max())
    accuracy = unrolled_fp64_error(eng, theta, Wp, labels, srcs, dsts, tabs, sides, S, T, batch)
    extra = {}
    if batch:
        losses = []
        opt = torch.optim.SGD([Wp], lr=0.1)
        t0 = time.perf_counter()
        for _ in range(50):
            opt.zero_grad()
            lb = eng(theta.detach(), Wp)
            loss = ce_loss(lb, labels)
            loss.backward()
            opt.step()
            losses.append(float(loss.item()))
        torch.cuda.synchronize()
        extra = {"sgd_steps": 50, "lr": 0.1, "loss_first": losses[0], "loss_last": losses[-1],
                 "sgd_ms_per_step": 1e3 * (time.perf_counter() - t0) / 50,
                 "networks_per_s_fwd_bwd": len(sides) / (fb_ms / 1e3)}
    eng.close()
    if rank != 0:
        return 0
    line = {"metric": "BP fwd+bwd ms", "value": fb_ms, "unit": "ms", "n_gpus": 1, "steps": reps,
            "warmup": a.warmup, "ms_per_step": fb_ms, "higher_is_better": False, "scaling": "replicas",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": (f"{len(sides)} grid MRFs, side U[32,256], " if batch else "512x512 grid MRF, ")
                       + f"{S} states, T={T}, checkpoints every 5, shared pairwise table",
                       "nodes": V, "edges": E},
            "forward_ms": f_ms, "fwd_bwd_over_fwd": fb_ms / f_ms, "plain_forward_ms": p_ms,
            "fwd_bwd_over_plain_forward": fb_ms / p_ms, "max_abs_belief_diff_vs_plain": max_diff,
            "max_abs_err_vs_fp64": accuracy["max_abs_err_vs_fp64"], "accuracy": accuracy,
            "clocks": clk, **extra}
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return run_reference_arm(a, rank, world)
    if a.workload == "batched":
        return run_batched(a, rank, world)
    if a.workload == "tree":
        return run_tree(a, rank, world)
    if a.workload == "random10k":
        return run_random10k(a, rank, world)
    if a.workload in ("unrolled", "unrolled_batch"):
        return run_unrolled(a, rank, world, a.workload == "unrolled_batch")

    import torch
    import belief_network_wrapper as W
    from belief_propagation_b200.engine import BPGraph

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    t0 = time.time()
    net = W.bp.synth.power_law_loopy(a.nodes, a.edges, 2, 0.10, seed=1)
    V, E, S = net.V, net.E, 2
    gen_s = time.time() - t0
    # a dedicated stream: the library's kernels, the CUDA graphs it captures
    # and the timing events all live on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    handle = stream.cuda_stream

    if a.shard:
        return run_sharded(a, rank, world, net, gen_s, dist, barrier, local)

    # ---- resident graph
    g = BPGraph(V, net.src, net.dst, net.joint, uniform_states=2, stream=handle, reorder=bool(a.reorder))
    prior = torch.from_numpy(net.beliefs).cuda()

    def step():
        g.set_beliefs(prior)
        g.init_messages()
        return g.loopy(0.0, a.iterations, delta="f64")

    for _ in range(a.warmup):
        step()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    kernel_ms = []
    for _ in range(a.steps):
        r = step()
        kernel_ms.append(r["elapsed_ms"] / max(r["executed"], 1))
    split = r["kernel_used"] == 4   # BP_KERNEL_SPLIT
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, dist)
    ms_per_step = ms / a.steps
    updates = float(E) * a.iterations * world
    value = updates / (ms_per_step / 1e3)

    # ---- roofline of one iteration: one k_flood launch, or the split
    # schedule's send pass + node pass (the library's choice for send buffers
    # larger than L2); its algorithmic bytes are the iteration's minimum
    it_ms = statistics.median(kernel_ms)
    algo = flood_bytes_per_iteration(V, E, S)
    achieved = algo / (it_ms / 1e3) / 1e9
    peak, peak_src = measured_hbm_peak()
    if split:
        traffic = profiled_traffic("k_flood_split_power_law_16M_dram.md", "traffic_bytes_per_iteration")
        kernel = "k_flood_send<2,0> + k_flood_nodes<2,0,1> (one split iteration, 2 launches)"
    else:
        traffic = profiled_traffic("k_flood_power_law_16M_dram.md")
        kernel = "k_flood<2,true>"
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": kernel, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": algo, "algorithmic_bytes_per_iteration": algo, "launch_ms": it_ms,
                "iteration_ms": it_ms, "launches_per_iteration": 2 if split else 1}
    graph_bytes = g.device_bytes()
    g.close()
    del prior
    torch.cuda.empty_cache()

    # ---- end to end through the C-ABI with host buffers
    e2e = None
    if not a.no_e2e:
        pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
        src_h, dst_h, joint_h, bel_h = pin(net.src), pin(net.dst), pin(net.joint), pin(net.beliefs)
        out_h = torch.empty((V, S), dtype=torch.float32).pin_memory()

        phases = {"create_ms": 0.0, "solve_ms": 0.0, "read_ms": 0.0, "destroy_ms": 0.0}
        # the serving loop's memory reservation, made once at start-up: room
        # for a graph solving, the next one building, its temporaries, and
        # slack for the pool's fragmentation
        from belief_propagation_b200 import native as N
        reserve = 6 * int(graph_bytes)
        if N.load().bp_reserve_cached_memory(reserve) != 0:
            # not enough free memory for the reservation: the loop runs
            # without one (and may see the pool's growth stalls)
            reserve = 0

        def e2e_step(record=False):
            t0 = time.perf_counter()
            g2 = BPGraph(V, src_h, dst_h, joint_h, uniform_states=2, stream=handle, reorder=bool(a.reorder))
            g2.set_beliefs(bel_h)
            t1 = time.perf_counter()
            g2.init_messages()
            g2.loopy(0.0, a.iterations, delta="f64")
            t2 = time.perf_counter()
            g2.beliefs(out=out_h)
            t3 = time.perf_counter()
            g2.close()
            t4 = time.perf_counter()
            if record:
                for k, dt in zip(phases, (t1 - t0, t2 - t1, t3 - t2, t4 - t3)):
                    phases[k] += 1e3 * dt / a.e2e_steps

        e2e_step()
        barrier()
        # one step after another: the phases of a step
        t0 = time.perf_counter()
        for _ in range(a.e2e_steps):
            e2e_step(record=True)
        barrier()
        seq_ms = (time.perf_counter() - t0) / a.e2e_steps * 1e3

        # pipelined, as a serving loop runs it: a second host thread builds
        # graph k+1 (pinned-host upload, device CSR build, beliefs) on its own
        # stream while this thread solves graph k and a third reads graph
        # k-1's beliefs back; every step's copies and work stay inside the
        # timed region, which runs from before the first build to after the
        # last read
        from concurrent.futures import ThreadPoolExecutor
        # equal stream priorities: a low-priority build starves for a whole
        # CUDA-graph chunk of the solve at each of its host synchronisations
        streams = [torch.cuda.Stream() for _ in range(3)]
        outs = [out_h, torch.empty((V, S), dtype=torch.float32).pin_memory()]

        def build(k):
            gk = BPGraph(V, src_h, dst_h, joint_h, uniform_states=2, stream=streams[k % 3].cuda_stream,
                         reorder=bool(a.reorder))
            gk.set_beliefs(bel_h)
            return gk

        def finish(gk, k):
            gk.beliefs(out=outs[k % 2])
            gk.close()

        def pipelined(n):
            # three host threads: this one solves graph k while one builds
            # graph k+1 and another reads graph k-1's beliefs back (device to
            # pinned host) and releases it; the run ends after the last read
            with ThreadPoolExecutor(max_workers=1) as ex, ThreadPoolExecutor(max_workers=1) as rd:
                fut = ex.submit(build, 0)
                reads = []
                for k in range(n):
                    gk = fut.result()
                    if k + 1 < n:
                        fut = ex.submit(build, k + 1)
                    gk.init_messages()
                    gk.loopy(0.0, a.iterations, delta="f64")
                    reads.append(rd.submit(finish, gk, k))
                for r in reads:
                    r.result()

        pipelined(2)
        barrier()
        # three timed runs of e2e_steps steps each; the median run is the number
        runs = []
        for _ in range(3):
            t0 = time.perf_counter()
            pipelined(a.e2e_steps)
            barrier()
            runs.append((time.perf_counter() - t0) / a.e2e_steps * 1e3)
        ems = max_over_ranks(sorted(runs)[1], dist)
        e2e = {"value": float(E) * a.iterations * world / (ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(E * (4 + 4 + 4 * S * S) + V * 4 * S), "d2h_bytes_per_step": int(V * 4 * S),
               "ms_per_step": ems, "steps": a.e2e_steps,
               "timing": "wall clock over all steps, first build included; median of 3 runs",
               "runs_ms_per_step": [round(r, 2) for r in runs],
               "pipelined": "the build of step k+1 (its H2D copies included) and the read-back of step k-1 overlap "
                            "the solve of step k",
               "sequential_ms_per_step": round(max_over_ranks(seq_ms, dist), 2),
               "pool_reserved_bytes": reserve,
               "phases_wall_ms": {k: round(v, 2) for k, v in phases.items()}}

    cpu = None
    accuracy = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            cpu = reference_sample()
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "unavailable", "sample": str(ex)[:200]}
        try:
            accuracy = power_law_accuracy(a, handle)
        except Exception as ex:  # reported, not fatal
            accuracy = {"error": str(ex)[:200]}

    others = None
    if rank == 0 and world == 1 and a.configs == "all":
        others = run_other_configs(a)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    # set_beliefs, init, gather, then flood x iterations, or (split) the
    # conversion to send order, 2 x iterations and the two conversions back
    launches_per_step = 3 + (3 + 2 * a.iterations if split else a.iterations)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(a), "nodes": V, "edges": E, "states": S,
                       "iterations": a.iterations, "l2": "inputs larger than L2 (working set ~3.4 GB per replica)",
                       "node_order": "renumbered by out-degree" if a.reorder else "caller ids",
                       "parallelism": f"replicas x{world}", "generator_s": round(gen_s, 1)},
            "hbm_gbs_algorithmic": achieved, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches_per_step * a.steps, "clocks": clk}
    if accuracy is not None:
        line.update({k: accuracy[k] for k in ("max_abs_err_vs_oracle", "max_abs_err_vs_fp64", "fp64_iterations")
                     if k in accuracy})
        line["accuracy"] = accuracy
    if others is not None:
        line["other_configs"] = others
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
