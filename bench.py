"""Benchmark of the cycle-search hot path on B200.

Workload (default): one shape pair on the GPU -- a perturbed genus-0 mesh X
with 5,000 vertices (both orientations of its ~30k edges) and normals, a
200-point closed silhouette curve Y with in-plane normals, 64-d float32
features -> feat_diff; conjugate product graph, k = 3, cost/time mode
("vanilla", "lengthnormalisation") [cost = feature difference, time = edge
length].  Inputs are seeded synthetic data of that shape (no dataset).

One step = recompute the edge costs on the device (generate) + one minimum
cost/time-ratio cycle solve (lawlergpu).  `value` is solves/s with the inputs
resident in HBM, timed with CUDA events on the solver's stream; `e2e` is the
same solve through the public API from host arrays (handle creation, host ->
device copies, template build, solve, matching read back).

--impl reference times the reference algorithm's CPU implementation (the
restatement under oracle/; the reference itself cannot be compiled in this
environment) on the host cores: a full lawlercpu solve during warm-up gives
the sweep count, each timed step times a bounded sample (one Bellman-Ford
sweep), and solves/s = 1 / (energy + rescale + in-edge sets + sweeps x sweep).

Multi-GPU: the path does not shard within a pair; --gpus N runs N independent
replicas (one pair per rank, seed = rank), value = total solves / max time.
"""
from __future__ import annotations

import os

# before anything starts CUDA: 32 host work queues let batched solves (one
# stream per pair) run side by side; the default of 8 serialises them
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import argparse
import gc
import json
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "product-graph-cycles_b200"))

METRIC = "ratio-cycle solves/s + fwd/bwd pairs/s, 1 B200, vs plain GPU Lawler; BF HBM GB/s"
L2_BYTES = 126 * 10**6  # B200 L2
WORKLOADS = {
    # name: (n_vertices, n_curve, feat_dim, conj, reg, prune, cost, time, k)
    "single_pair_conj_5k_200_k3": (5000, 200, 64, True, False, False, "vanilla", "lengthnormalisation", 3),
    "plain_642_60_k2": (642, 60, 32, False, False, False, "vanilla", "nomode", 2),
    # smaller conjugate pair used for ncu captures (inputs still larger than L2)
    "conj_2k_100_k3": (2000, 100, 64, True, False, False, "vanilla", "lengthnormalisation", 3),
    # large pair at the HBM-bound scale: conjugate + pruned, SO(3) robust cost against feature time
    "conj_prune_20k_500_k4": (20000, 500, 64, True, True, True, "robustso3", "feature", 4),
    # the same layer with 100 layers: ncu captures of the large pair's steps (about 3 GB on the device)
    "conj_prune_20k_100_k4": (20000, 100, 64, True, True, True, "robustso3", "feature", 4),
}
DEFAULT_WORKLOAD = "single_pair_conj_5k_200_k3"
# batched serving: many plain pairs of uneven size solved concurrently
BATCHES = {
    # name: (pairs, |VX| range, |VY| range (even), k choices, feature dim)
    "batch_256_plain_1k8k": (256, (1000, 8000), (50, 250), (2, 3), 32),
}
# differentiation: forward (batched ratio solves) + backward (adjoint kernel) to learnable features
FWDBWD = {
    # name: (pairs, |VX|, |VY|, k, feature dim)
    "fwdbwd_32_plain_2k_100_k2": (32, 2000, 100, 2, 64),
}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _make_pair(name, seed):
    from cyclic_product_graphs import synthetic

    nv, ny, dim, conj, reg, prune, cost, tme, k = WORKLOADS[name]
    if name.startswith("plain_642"):
        p = synthetic.make_pair(icosphere_level=3, n_curve=ny, feat_dim=dim, seed=seed)
    else:
        p = synthetic.make_pair(n_vertices=nv, n_curve=ny, feat_dim=dim, seed=seed)
    return p, dict(conj=conj, reg=reg, prune=prune, cost=cost, time=tme, k=k)


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.at_end = False

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if not self.lines:
            # a timed region shorter than the sampling period: one query at
            # its end, while the clocks still reflect the load
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=10)
                self.lines += [x.strip() for x in out.stdout.splitlines() if x.strip()]
                self.at_end = True
            except Exception:
                pass

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}
        if self.at_end:
            out["note"] = "timed region shorter than the 200 ms sampling period: sampled at its end"
        return out


def _dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value, world, device):
    """The largest `value` of all ranks (every rank gets it); `value` itself at one rank."""
    if world <= 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(solves_per_rank, world, max_ms):
    """Whole-job solves/s of `world` replicas that each ran `solves_per_rank` solves, timed as the max over ranks."""
    return world * solves_per_rank / (max_ms / 1000.0)


def algorithmic_bytes_per_sweep(info, k, ratio_mode):
    """Bytes one Bellman-Ford sweep must move: (4 + 4c)(E_inter + (K-1) E_intra) + 8 K n (nY + 1).

    Every interlayer edge is visited once per sweep and every intralayer edge
    once per depth 1..K-1; a visit reads the int32 source index and c fp32
    cost columns (c = 2 in ratio mode with a time column, else 1).  Every
    (node, depth) of the nY + 1 layers writes an fp32-sized value and an
    int32 predecessor.  Gathered source values are not counted.  Without
    intralayer edges (pruned graphs) only depth 0 of each layer is ever
    reached, so K is replaced by 1 in the node term.
    """
    L = info["layers"]
    c = 2 if (ratio_mode and info["cost_columns"] > 1) else 1
    e_inter = L * info["inter_edges_per_layer"]
    e_intra = L * info["intra_edges_per_layer"]
    nodes = info["nodes_per_layer"] * (L + 1)
    depths = k if e_intra > 0 else 1
    return (4 + 4 * c) * (e_inter + (k - 1) * e_intra) + 8 * depths * nodes


def run_ours(args, world, rank):
    import numpy as np
    import torch

    import cyclic_product_graphs as cpg

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dev = torch.cuda.current_device()
    pair, cfg = _make_pair(args.workload, seed=args.seed + rank)
    k = cfg["k"]
    hargs = (pair["VX"], pair["EX"], pair["VY"], pair["EY"], pair["feat_diff"], cfg["conj"], cfg["reg"], cfg["prune"])

    g = cpg.product_graph_generator(*hargs)
    if cfg["conj"]:
        g.set_normals(pair["NX"], pair["NY"])
    g.set_cost_time_ratio_mode(cfg["cost"], cfg["time"])
    stream = torch.cuda.Stream()
    g.set_stream(stream.cuda_stream)
    g.generate()
    info = g.graph_info()

    def step():
        g.generate()
        return g.solve_with_cost_time_ratio("lawlergpu", k)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sweeps = bf_us = launches = 0
    result = None
    # cost streams smaller than L2 (126 MB): flush L2 between the timed steps
    # with a 256 MB write on the solver's stream, outside the steps' events
    edges = info["layers"] * info["edges_per_block"]
    flush = torch.empty(1 << 25, dtype=torch.float64, device="cuda") if 8 * edges < L2_BYTES else None
    with ClockSampler(dev) as clocks:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(args.steps):
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.fill_(float(i))
            ev[i][0].record(stream)
            result = step()
            ev[i][1].record(stream)
            st = g.last_stats()
            prof = g.last_profile()
            last_sweeps = st["sweeps"]
            sweeps += st["sweeps"]
            bf_us += st["device_us"]
            launches += st["kernel_launches"] + 1  # + the energy kernel of generate()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(sum(step_ms), world, "cuda")
    ms_per_step = total_ms / args.steps
    value = replica_throughput(args.steps, world, total_ms)

    # roofline of the dominant kernel (the Bellman-Ford launch)
    peak, peak_kind = _peaks()
    b_sweep = algorithmic_bytes_per_sweep(info, k, True)
    achieved = (b_sweep * sweeps) / (bf_us * 1e-6) / 1e9 if bf_us else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", f"bf_kernel_{args.workload}.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                traffic = json.load(f).get("dram_bytes_per_launch")
        except Exception:
            traffic = None

    # End to end through the public API from host buffers, as a serving
    # process runs it: one fresh handle per request, created after the timed
    # handle has been released (as in the batch and fwd/bwd workloads; a live
    # second handle made each request ~4 ms slower on the host).
    del g
    gc.collect()
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    h2d = sum(int(np.asarray(pair[key]).nbytes) for key in ("VX", "EX", "VY", "EY", "feat_diff"))
    if cfg["conj"]:
        h2d += int(pair["NX"].nbytes + pair["NY"].nbytes)
    d2h = 0
    for it in range(e2e_steps + 1):  # the first pass is an untimed warm-up (module loading, first allocations)
        if it == 1:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
        ge = cpg.product_graph_generator(*hargs)
        if cfg["conj"]:
            ge.set_normals(pair["NX"], pair["NY"])
        ge.set_cost_time_ratio_mode(cfg["cost"], cfg["time"])
        out = ge.solve_with_cost_time_ratio("lawlergpu", k)
        d2h = int(out[2].nbytes) + 8
        del ge
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_value = world * e2e_steps / e2e_s

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 (fp32 integer-valued cost streams)",
        "data": "synthetic (seeded)",
        "config": _pair_config(args.workload, cfg, info["nodes_per_layer"], info["layers"],
                               info["layers"] * info["edges_per_block"], world),
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_kind": f"{peak_kind} hbm_gbs", "kernel": "bf_kernel",
                     "algorithmic_bytes_per_sweep": b_sweep, "sweeps_per_solve": sweeps / args.steps,
                     "bf_ms_per_solve": bf_us / 1000.0 / args.steps},
        "bf_team": {"ctas": prof["ctas"], "threads": prof["threads"], "wait_list_entries": prof["wait_entries"],
                    "cycles_per_step": {key[7:]: round(prof[key] / max(1, prof["steps"]), 1)
                                        for key in ("cycles_relax", "cycles_stage_wait", "cycles_handoff",
                                                    "cycles_bookkeeping", "cycles_sweep_tail")},
                    "tail_cycles_per_sweep": {key[12:]: round(prof[key] / max(1, last_sweeps), 1)
                                              for key in ("cycles_tail_wrap", "cycles_tail_candidates",
                                                          "cycles_tail_lead")},
                    "last_solve": {key: st[key] for key in ("bf_calls", "sweeps", "candidates", "fallback_walks",
                                                            "lawler_iters")}},
        "clocks": clocks.summary(),
        "result": {"objective": result[1], "cycle_edges": int(result[2].shape[0])},
        "wall_s": wall,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(pair, cfg, sweeps / args.steps, args.cpu_sweeps)
    return line


def cpu_baseline(pair, cfg, sweeps_per_solve, sample_sweeps):
    """The reference algorithm on the host cores: measured phases of one ratio
    solve, with `sample_sweeps` Bellman-Ford sweeps timed and scaled to the
    solve's sweep count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    cores = os.cpu_count() or 1
    orc.set_threads(cores)
    hargs = (pair["VX"], pair["EX"], pair["VY"], pair["EY"], pair["feat_diff"], cfg["conj"], cfg["reg"], cfg["prune"])
    o = orc.OracleGenerator(*hargs)
    if cfg["conj"]:
        o.set_normals(pair["NX"], pair["NY"])
    o.set_cost_time_ratio_mode(cfg["cost"], cfg["time"])
    t0 = time.perf_counter()
    o.generate()
    t_gen = time.perf_counter() - t0
    ph = o.time_phases(cfg["k"], 0.3, sample_sweeps)
    t_solve = ph["energy_s"] + ph["rescale_s"] + ph["in_graph_s"] + sweeps_per_solve * ph["sweep_s"]
    return {"value": 1.0 / t_solve, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": (f"oracle lawlercpu restatement, OpenMP x{cores}: energy {ph['energy_s']:.2f}s + rescale "
                       f"{ph['rescale_s']:.2f}s + in-edge sets {ph['in_graph_s']:.2f}s measured, "
                       f"{sample_sweeps} Bellman-Ford sweeps timed ({ph['sweep_s']:.3f}s each) and scaled to "
                       f"{sweeps_per_solve:.1f} sweeps/solve; product-graph build {t_gen:.1f}s not counted"),
            "phases_s": ph}


def _pair_config(workload, cfg, nodes_per_layer, layers, edges, world):
    """The `config` of a single-pair line, the same in both arms."""
    l2 = ("inputs larger than L2 (fp64 cost stream > 126 MB)" if 8 * edges >= L2_BYTES
          else "L2 flushed between timed steps (256 MB write; the cost streams are smaller than L2)")
    return {"workload": workload, "k": cfg["k"], "nodes_per_layer": int(nodes_per_layer), "layers": int(layers),
            "edges": int(edges), "cost_mode": [cfg["cost"], cfg["time"]], "parallelism": f"replicas x{world}",
            "l2": l2}


def run_reference(args):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    pair, cfg = _make_pair(args.workload, seed=args.seed)
    cores = os.cpu_count() or 1
    orc.set_threads(cores)
    hargs = (pair["VX"], pair["EX"], pair["VY"], pair["EY"], pair["feat_diff"], cfg["conj"], cfg["reg"], cfg["prune"])
    o = orc.OracleGenerator(*hargs)
    if cfg["conj"]:
        o.set_normals(pair["NX"], pair["NY"])
    o.set_cost_time_ratio_mode(cfg["cost"], cfg["time"])
    o.generate()
    # warm-up: one full solve fixes the sweep count of a solve, one timed
    # pass of the per-solve phases (energy, rescale, in-edge sets) their cost
    t0 = time.perf_counter()
    res = o.solve_with_cost_time_ratio("lawlercpu", cfg["k"])
    t_full = time.perf_counter() - t0
    stats = o.last_stats()
    sweeps = stats["sweeps"]
    ph = o.time_phases(cfg["k"], 0.3, 1)
    fixed = ph["energy_s"] + ph["rescale_s"] + ph["in_graph_s"]
    for _ in range(max(0, args.warmup - 1)):
        o.time_sweeps(cfg["k"], 0.3, 1)
    # timed steps: one Bellman-Ford sweep each (the bounded sample)
    samples = [o.time_sweeps(cfg["k"], 0.3, 1) for _ in range(args.steps)]
    sweep_s = statistics.median(samples)
    t_solve = fixed + sweeps * sweep_s
    value = 1.0 / t_solve
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * t_solve, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": _pair_config(args.workload, cfg, 3 * len(pair["EX"]) if cfg["conj"] else len(pair["VX"]),
                               len(pair["EY"]), o.product_space_rows(), int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"one Bellman-Ford sweep per step (median {sweep_s:.3f}s) scaled to {sweeps} "
                                   f"sweeps/solve, plus energy {ph['energy_s']:.2f}s + rescale {ph['rescale_s']:.2f}s "
                                   f"+ in-edge sets {ph['in_graph_s']:.2f}s timed once; a full warm-up solve took "
                                   f"{t_full:.1f}s"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "full_solve_s": t_full, "result": {"objective": res[1], "cycle_edges": int(res[2].shape[0])},
    }


def _batch_specs(name, seed):
    import numpy as np

    count, (v0, v1), (m0, m1), ks, dim = BATCHES[name]
    rng = np.random.default_rng(seed)
    return [dict(nv=int(rng.integers(v0, v1 + 1)), m=2 * int(rng.integers(m0 // 2, m1 // 2 + 1)),
                 k=int(rng.choice(ks)), dim=dim, seed=seed * 100000 + i) for i in range(count)]


def _batch_pair(spec):
    sys.path.insert(0, os.path.join(ROOT, "product-graph-cycles_b200"))
    from cyclic_product_graphs import synthetic

    p = synthetic.make_pair(n_vertices=spec["nv"], n_curve=spec["m"], feat_dim=spec["dim"], seed=spec["seed"],
                            with_normals=False)
    return {k: p[k] for k in ("VX", "EX", "VY", "EY", "feat_diff")}


def _batch_config(workload, pairs, world):
    """The `config` of a batch line, the same in both arms.  A plain block
    holds 2|EX| + |VX| edges (an intra- and an interlayer copy of every X
    edge, and the vertical edges), so the total is known from the inputs."""
    return {"workload": workload, "pairs": len(pairs), "vx_range": BATCHES[workload][1],
            "vy_range": BATCHES[workload][2], "k": BATCHES[workload][3],
            "edges_total": int(sum(len(p["EY"]) * (2 * len(p["EX"]) + len(p["VX"])) for p in pairs)),
            "parallelism": f"one stream + a small CTA team per pair, replicas x{world}",
            "l2": "inputs larger than L2 (all pairs' cost streams together)"}


def _fwdbwd_config(workload, pairs, k, world):
    """The `config` of a fwd/bwd line, the same in both arms."""
    return {"workload": workload, "pairs": int(pairs), "vx": FWDBWD[workload][1], "vy": FWDBWD[workload][2],
            "k": int(k), "feature_dim": FWDBWD[workload][4],
            "parallelism": f"one stream + a small CTA team per pair, replicas x{world}",
            "l2": "per-pair streams of all pairs exceed L2"}


def _batch_pairs(name, seed):
    """The batch's seeded pairs, built in parallel host processes (spawned, before any GPU work)."""
    import multiprocessing as mp

    specs = _batch_specs(name, seed)
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        pairs = pool.map(_batch_pair, specs, chunksize=4)
    return specs, pairs


def run_batch(args, world, rank):
    """Batched serving: every step solves all pairs of the batch concurrently
    (solve_batch: one stream and a small Bellman-Ford team per pair, the teams
    the device runs side by side covering its SMs; costs regenerated on the
    device first).  Also timed: the same pairs solved one
    after the other with full-GPU teams (the plain per-pair GPU Lawler)."""
    specs, pairs = _batch_pairs(args.workload, args.seed + rank)
    import numpy as np
    import torch

    import cyclic_product_graphs as cpg

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dev = torch.cuda.current_device()

    def make(i):
        p = pairs[i]
        g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, False)
        g.set_cost_time_ratio_mode("vanilla", "nomode")
        g.set_max_depth_cost_time_ratio(specs[i]["k"])
        return g

    gens = [make(i) for i in range(len(pairs))]
    for g in gens:
        g.generate()
    infos = [g.graph_info() for g in gens]

    def step():
        return cpg.solve_batch(gens, "lawlergpu", None, regenerate=True)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    bytes_moved = 0
    with ClockSampler(dev) as clocks:
        for i in range(args.steps):
            torch.cuda.synchronize()
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
            torch.cuda.synchronize()
            for g, info, sp in zip(gens, infos, specs):
                bytes_moved += algorithmic_bytes_per_sweep(info, sp["k"], True) * g.last_stats()["sweeps"]
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world, "cuda")
    solves = len(gens) * args.steps
    value = replica_throughput(solves, world, total_ms)
    peak, peak_kind = _peaks()
    achieved = bytes_moved / (total_ms * 1e-3) / 1e9

    # the plain per-pair GPU Lawler: the same pairs one after the other, full-GPU teams
    seq_n = len(gens)
    for g in gens[:seq_n]:
        g.generate()
        g.solve_with_cost_time_ratio("lawlergpu")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for g in gens[:seq_n]:
        g.generate()
        g.solve_with_cost_time_ratio("lawlergpu")
    e1.record(stream)
    torch.cuda.synchronize()
    seq_value = seq_n / (e0.elapsed_time(e1) / 1000.0)

    # end to end from host arrays: handles built, batch solved, matchings back
    # (the timed handles are released first: their memory returns to the
    # library's caching allocator, as in a serving process)
    launches = sum(g.last_stats()["kernel_launches"] + 1 for g in gens)
    del gens
    import gc

    gc.collect()
    h2d = sum(int(sum(np.asarray(p[k]).nbytes for k in p)) for p in pairs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fresh = [make(i) for i in range(len(pairs))]
    results = cpg.solve_batch(fresh, "lawlergpu", None)
    e2e_s = time.perf_counter() - t0
    d2h = sum(int(r[2].nbytes) + 8 for r in results)
    del fresh

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (fp32 integer-valued cost streams)", "data": "synthetic (seeded)",
        "config": _batch_config(args.workload, pairs, world),
        "vs_plain_gpu_lawler": {"plain_solves_per_s": seq_value, "ratio": value / seq_value,
                                "sample": f"all {seq_n} pairs solved one after the other, full-GPU teams"},
        "e2e": {"value": world * len(pairs) / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": 1},
        "gpu_launches": None,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": f"{peak_kind} hbm_gbs", "kernel": "bf_kernel (all pairs)",
                     "note": "algorithmic bytes of every sweep of every pair / batch step time"},
        "clocks": clocks.summary(),
    }
    line["gpu_launches"] = launches * args.steps
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = _batch_cpu_sample(specs, pairs)
    return line


def _batch_cpu_sample(specs, pairs, count=2):
    """The oracle's lawlercpu on the first `count` pairs of the batch, all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    cores = os.cpu_count() or 1
    orc.set_threads(cores)
    t = 0.0
    for spec, p in zip(specs[:count], pairs[:count]):
        o = orc.OracleGenerator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, False)
        o.set_cost_time_ratio_mode("vanilla", "nomode")
        t0 = time.perf_counter()
        o.generate()
        o.solve_with_cost_time_ratio("lawlercpu", spec["k"])
        t += time.perf_counter() - t0
    return {"value": count / t, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"oracle generate + lawlercpu, OpenMP x{cores}, on the batch's first {count} pairs "
                      f"({[(s['nv'], s['m'], s['k']) for s in specs[:count]]}), solved one after the other"}


def run_reference_batch(args):
    specs, pairs = _batch_pairs(args.workload, args.seed)
    samples = []
    for _ in range(max(0, args.warmup - 1)):
        _batch_cpu_sample(specs, pairs, 1)
    for i in range(args.steps):
        samples.append(_batch_cpu_sample(specs[i % len(specs):], pairs[i % len(pairs):], 1)["value"])
    value = statistics.median(samples)
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": _batch_config(args.workload, pairs, int(os.environ.get("WORLD_SIZE", "1"))),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": "port",
                             "sample": "oracle generate + lawlercpu of one pair of the batch per step "
                                       "(pairs 0..steps-1), median"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _fwdbwd_pairs(name, seed):
    count, nv, m, k, dim = FWDBWD[name]
    specs = [dict(nv=nv, m=m, k=k, dim=dim, seed=seed * 100000 + i) for i in range(count)]
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        pairs = pool.map(_fwdbwd_pair, specs)
    return specs, pairs


def _fwdbwd_pair(spec):
    sys.path.insert(0, os.path.join(ROOT, "product-graph-cycles_b200"))
    from cyclic_product_graphs import synthetic

    p = synthetic.make_pair(n_vertices=spec["nv"], n_curve=spec["m"], feat_dim=spec["dim"], seed=spec["seed"],
                            with_normals=False)
    return {k: p[k] for k in ("VX", "EX", "VY", "EY", "feat_diff", "fX", "fY")}


def run_fwdbwd(args, world, rank):
    """Forward + backward: feat_diff = ||f_X - f_Y|| from learnable float32
    features (torch), lambda* of every pair by one batched ratio solve, and
    d(sum lambda*)/d features through the adjoint kernel and torch.  Also
    timed: the same pairs one after the other with full-GPU teams (the plain
    per-pair GPU Lawler, forward + backward)."""
    specs, pairs = _fwdbwd_pairs(args.workload, args.seed + rank)
    import numpy as np
    import torch

    import cyclic_product_graphs as cpg
    from cyclic_product_graphs.autograd import RatioCycleObjective, ratio_cycle_objectives

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dev = torch.cuda.current_device()
    k = specs[0]["k"]

    def make(p):
        g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, False)
        g.set_cost_time_ratio_mode("vanilla", "nomode")
        return g

    gens = [make(p) for p in pairs]
    fX = [torch.tensor(p["fX"], device="cuda", requires_grad=True) for p in pairs]
    fY = [torch.tensor(p["fY"], device="cuda", requires_grad=True) for p in pairs]

    def step():
        fds = [torch.cdist(a, b).double() for a, b in zip(fX, fY)]
        lam = ratio_cycle_objectives(gens, fds, k)
        lam.sum().backward()
        return lam

    def step_plain():
        for g, a, b in zip(gens, fX, fY):
            g.set_team_cap(0)
            RatioCycleObjective.apply(torch.cdist(a, b).double(), g, k).backward()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(dev) as clocks:
        for i in range(args.steps):
            torch.cuda.synchronize()
            ev[i][0].record(stream)
            lam = step()
            ev[i][1].record(stream)
            torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world, "cuda")
    value = replica_throughput(len(gens) * args.steps, world, total_ms)
    grads_ok = all(t.grad is not None and bool(torch.isfinite(t.grad).all()) for t in fX)

    step_plain()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    step_plain()
    e1.record(stream)
    torch.cuda.synchronize()
    plain_value = len(gens) / (e0.elapsed_time(e1) / 1000.0)

    # end to end: host features -> device, fresh handles, forward + backward, gradients back to the host
    # (the timed handles are released first, as in a serving process)
    mean_objective = float(lam.detach().mean())
    del gens, lam
    import gc

    gc.collect()
    h2d = sum(int(p[k2].nbytes) for p in pairs for k2 in ("VX", "EX", "VY", "EY", "fX", "fY"))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fresh = [make(p) for p in pairs]
    ax = [torch.from_numpy(p["fX"]).pin_memory().to("cuda", non_blocking=True).requires_grad_(True) for p in pairs]
    by = [torch.from_numpy(p["fY"]).pin_memory().to("cuda", non_blocking=True) for p in pairs]
    lam_e = ratio_cycle_objectives(fresh, [torch.cdist(a, b).double() for a, b in zip(ax, by)], k)
    lam_e.sum().backward()
    host_grads = [a.grad.cpu() for a in ax]
    e2e_s = time.perf_counter() - t0
    d2h = sum(int(gr.numel() * gr.element_size()) for gr in host_grads) + 8 * len(pairs)

    return {
        "metric": METRIC, "value": value, "unit": "fwd+bwd pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 solve / fp32 features", "data": "synthetic (seeded)",
        "config": _fwdbwd_config(args.workload, len(pairs), k, world),
        "vs_plain_gpu_lawler": {"plain_pairs_per_s": plain_value, "ratio": value / plain_value,
                                "sample": "the same pairs, forward + backward one after the other, full-GPU teams"},
        "e2e": {"value": world * len(pairs) / e2e_s, "unit": "fwd+bwd pairs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": 1},
        "gradients_finite": grads_ok,
        "mean_objective": mean_objective,
        "gpu_launches": None,
        "clocks": clocks.summary(),
    }


def run_reference_fwdbwd(args):
    """The oracle's lawlercpu (forward) on one pair per step; the reference has no backward."""
    specs, pairs = _fwdbwd_pairs(args.workload, args.seed)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    orc.set_threads(os.cpu_count() or 1)
    samples = []
    for i in range(args.warmup + args.steps):
        p = pairs[i % len(pairs)]
        o = orc.OracleGenerator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, False)
        o.set_cost_time_ratio_mode("vanilla", "nomode")
        t0 = time.perf_counter()
        o.generate()
        o.solve_with_cost_time_ratio("lawlercpu", specs[0]["k"])
        if i >= args.warmup:
            samples.append(time.perf_counter() - t0)
    value = 1.0 / statistics.median(samples)
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "fwd+bwd pairs/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": _fwdbwd_config(args.workload, len(specs), specs[0]["k"], int(os.environ.get("WORLD_SIZE", "1"))),
            "cpu_baseline": {"value": value, "unit": "fwd+bwd pairs/s", "cores": os.cpu_count() or 1, "kind": "port",
                             "sample": "oracle generate + lawlercpu of one pair per step (forward only: the "
                                       "reference has no backward), median"},
            "e2e": {"value": value, "unit": "fwd+bwd pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + sorted(BATCHES) + sorted(FWDBWD),
                    default=DEFAULT_WORKLOAD)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-sweeps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = _dist_env()

    if args.impl == "reference":
        if rank == 0:
            fn = run_reference_batch if args.workload in BATCHES else run_reference_fwdbwd \
                if args.workload in FWDBWD else run_reference
            print(json.dumps(fn(args)), flush=True)
        return

    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload in BATCHES:
        line = run_batch(args, world, rank)
    elif args.workload in FWDBWD:
        line = run_fwdbwd(args, world, rank)
    else:
        line = run_ours(args, world, rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
