"""Benchmark of the cycle-search hot path on B200.

The default run measures the whole metric ("ratio-cycle solves/s + fwd/bwd
pairs/s, 1 B200, vs plain GPU Lawler; BF HBM GB/s") and prints ONE JSON line:

* top level -- the single-pair GPU configuration: a perturbed genus-0 mesh X
  with 5,000 vertices (both orientations of its ~30k edges) and normals, a
  200-point closed silhouette curve Y with in-plane normals, 64-d float32
  features -> feat_diff; conjugate product graph, k = 3, cost/time mode
  ("vanilla", "lengthnormalisation").  One step = recompute the edge costs on
  the device (generate) + one minimum cost/time-ratio cycle solve
  (lawlergpu).  Its "dijkstragpu" sub-object times the minimum-cost solve of
  the same graph (generate + dijkstragpu per step).
* "configs" -- the other GPU configurations, each with its own value, e2e,
  roofline and (where the metric asks for it) vs_plain_gpu_lawler:
  batched serving of 256 uneven plain pairs, forward + backward on 32 plain
  pairs, and the large pruned conjugate pair (20k vertices x 500 curve
  points, k = 4).

`value` is throughput with the inputs resident in HBM, timed with CUDA
events on the solver's stream; `e2e` is the same work through the public API
from host arrays (handle creation, host -> device copies, template build,
solve, results back).  Inputs are seeded synthetic data of the stated shapes
(no dataset).  --workload NAME measures one configuration alone.

--impl reference times the reference algorithm's CPU implementation (the
restatement under oracle/; the reference itself cannot be compiled in this
environment) on all host cores, on the same configuration: every timed step
is one complete lawlercpu solve (energies recomputed on the product graph,
in-place rescale, in-edge sets, branch and bound), as many as fit a fixed
time budget; the line's `steps` is the number actually timed.

Multi-GPU: the path does not shard within a pair; --gpus N runs N independent
replicas (one pair per rank, seed = rank), value = total solves / max time.
"""
from __future__ import annotations

import os
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


def host_cpu():
    """The host's CPU model and the cores this process may use (lscpu's model name and affinity)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count() or 1
    return {"model": model, "usable_cores": usable, "logical_cpus": os.cpu_count() or 1}


def _solve_once(g, solver, k):
    return g.solve_with_cost_time_ratio("lawlergpu", k) if solver == "ratio" else \
        g.solve_with_minimum_cost("dijkstragpu", k)


def _time_pair_steps(g, stream, solver, k, steps, warmup, info, world):
    """Warm-up, then `steps` timed steps of generate + solve on `stream`
    (CUDA events around each step); the L2 is flushed between timed steps
    when the cost streams fit in it.  Returns the timing and counters."""
    import torch

    def step():
        g.generate()
        return _solve_once(g, solver, k)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    sweeps = bf_us = launches = 0
    result = st = prof = None
    edges = info["layers"] * info["edges_per_block"]
    flush = torch.empty(1 << 25, dtype=torch.float64, device="cuda") if 8 * edges < L2_BYTES else None
    import cyclic_product_graphs as cpg

    with ClockSampler(torch.cuda.current_device()) as clocks:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n0 = cpg.kernel_launches()
        for i in range(steps):
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.fill_(float(i))
            ev[i][0].record(stream)
            result = step()
            ev[i][1].record(stream)
            st = g.last_stats()
            prof = g.last_profile()
            sweeps += st["sweeps"]
            bf_us += st["device_us"]
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        launches = cpg.kernel_launches() - n0  # the library's kernels in the timed steps
    step_ms = [a.elapsed_time(b) for a, b in ev]
    return dict(total_ms=max_over_ranks(sum(step_ms), world, "cuda"), sweeps=sweeps, bf_us=bf_us,
                launches=launches, result=result, stats=st, profile=prof, clocks=clocks.summary(), wall=wall)


def _e2e_pair(cpg, hargs, pair, cfg, solver, steps, world):
    """The same solve end to end from host arrays: one fresh handle per
    request (created after the timed handle was released, as in a serving
    process), normals and modes set, solved, the matching read back."""
    import numpy as np
    import torch

    h2d = sum(int(np.asarray(pair[key]).nbytes) for key in ("VX", "EX", "VY", "EY", "feat_diff"))
    if cfg["conj"]:
        h2d += int(pair["NX"].nbytes + pair["NY"].nbytes)
    d2h = 0
    for it in range(steps + 1):  # the first pass is an untimed warm-up (module loading, first allocations)
        if it == 1:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
        ge = cpg.product_graph_generator(*hargs)
        if cfg["conj"]:
            ge.set_normals(pair["NX"], pair["NY"])
        ge.set_cost_time_ratio_mode(cfg["cost"], cfg["time"])
        out = _solve_once(ge, solver, cfg["k"])
        d2h = int(out[2].nbytes) + 8
        del ge
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    return {"value": world * steps / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps}


def _traffic(workload):
    """DRAM bytes of one Bellman-Ford launch of `workload` from its ncu summary under profiles/, and how it was got."""
    tpath = os.path.join(ROOT, "profiles", f"bf_kernel_{workload}.json")
    if not os.path.exists(tpath):
        return None, None
    try:
        with open(tpath) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch"), {"kind": d.get("kind", "unstated"), "source": d.get("source", "")}
    except Exception:
        return None, None


def measure_pair(args, world, rank, workload, steps, warmup, e2e_steps, with_min_cost=False, with_cpu=False):
    """One shape pair: ratio solves (and optionally min-cost solves) timed on
    the device, end to end through the public API, roofline of the
    Bellman-Ford kernel, and optionally the CPU baseline."""
    import torch

    import cyclic_product_graphs as cpg

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    pair, cfg = _make_pair(workload, seed=args.seed + rank)
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
    peak, peak_kind = _peaks()

    def roofline(t, ratio_mode, steps_done):
        b_sweep = algorithmic_bytes_per_sweep(info, k, ratio_mode)
        achieved = (b_sweep * t["sweeps"]) / (t["bf_us"] * 1e-6) / 1e9 if t["bf_us"] else None
        r = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
             "frac": (achieved / peak) if achieved else None, "traffic": None,
             "peak_kind": f"{peak_kind} hbm_gbs", "kernel": "bf_kernel",
             "algorithmic_bytes_per_sweep": b_sweep, "sweeps_per_solve": t["sweeps"] / steps_done,
             "bf_ms_per_solve": t["bf_us"] / 1000.0 / steps_done}
        if ratio_mode:
            r["traffic"], src = _traffic(workload)
            if src:
                r["traffic_kind"], r["traffic_source"] = src["kind"], src["source"]
        return r

    t = _time_pair_steps(g, stream, "ratio", k, steps, warmup, info, world)
    prof, st = t["profile"], t["stats"]
    line = {
        "metric": METRIC,
        "value": replica_throughput(steps, world, t["total_ms"]),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": t["total_ms"] / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 (fp32 integer-valued cost streams)",
        "data": "synthetic (seeded)",
        "config": _pair_config(workload, cfg, info["nodes_per_layer"], info["layers"],
                               info["layers"] * info["edges_per_block"], world),
        "gpu_launches": t["launches"],
        "roofline": roofline(t, True, steps),
        "bf_team": {"ctas": prof["ctas"], "threads": prof["threads"], "wait_list_entries": prof["wait_entries"],
                    "cycles_per_step": {key[7:]: round(prof[key] / max(1, prof["steps"]), 1)
                                        for key in ("cycles_relax", "cycles_stage_wait", "cycles_handoff",
                                                    "cycles_bookkeeping", "cycles_sweep_tail")},
                    "tail_cycles_per_sweep": {key[12:]: round(prof[key] / max(1, st["sweeps"]), 1)
                                              for key in ("cycles_tail_wrap", "cycles_tail_candidates",
                                                          "cycles_tail_lead")},
                    "last_solve": {key: st[key] for key in ("bf_calls", "sweeps", "candidates", "fallback_walks",
                                                            "lawler_iters")}},
        "clocks": t["clocks"],
        "result": {"objective": t["result"][1], "cycle_edges": int(t["result"][2].shape[0])},
        "wall_s": t["wall"],
    }
    if with_min_cost:
        tm = _time_pair_steps(g, stream, "min_cost", k, steps, warmup, info, world)
        line["dijkstragpu"] = {
            "value": replica_throughput(steps, world, tm["total_ms"]), "unit": "solves/s",
            "ms_per_step": tm["total_ms"] / steps, "steps": steps, "warmup": warmup,
            "gpu_launches": tm["launches"], "roofline": roofline(tm, False, steps), "clocks": tm["clocks"],
            "result": {"objective": tm["result"][1], "cycle_edges": int(tm["result"][2].shape[0]),
                       "bf_calls": tm["stats"]["bf_calls"], "branches": tm["stats"]["branches"]},
        }
    del g
    gc.collect()
    torch.cuda.synchronize()
    line["e2e"] = _e2e_pair(cpg, hargs, pair, cfg, "ratio", max(1, min(steps, e2e_steps)), world)
    if with_min_cost:
        line["dijkstragpu"]["e2e"] = _e2e_pair(cpg, hargs, pair, cfg, "min_cost", max(1, min(steps, e2e_steps)),
                                               world)
    cpg.release_cached_memory()
    if with_cpu and rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline(pair, cfg)
    return line


def _oracle_pair(orc, pair, cfg):
    hargs = (pair["VX"], pair["EX"], pair["VY"], pair["EY"], pair["feat_diff"], cfg["conj"], cfg["reg"], cfg["prune"])
    o = orc.OracleGenerator(*hargs)
    if cfg["conj"]:
        o.set_normals(pair["NX"], pair["NY"])
    o.set_cost_time_ratio_mode(cfg["cost"], cfg["time"])
    return o


def _oracle_step(o, solver, k):
    """One complete CPU step, the counterpart of the device's generate + solve:
    the energies recomputed on the product graph already built, then the
    whole lawlercpu (rescale, in-edge sets, branch and bound) or dijkstracpu
    solve."""
    t0 = time.perf_counter()
    o.recompute_energy()
    res = o.solve_with_cost_time_ratio("lawlercpu", k) if solver == "ratio" else \
        o.solve_with_minimum_cost("dijkstracpu", k)
    return time.perf_counter() - t0, res


def cpu_baseline(pair, cfg):
    """The reference algorithm on the host cores: one complete ratio step
    (energies + lawlercpu solve), timed once."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    cpu = host_cpu()
    orc.set_threads(cpu["usable_cores"])
    o = _oracle_pair(orc, pair, cfg)
    t0 = time.perf_counter()
    o.generate()
    t_graph = time.perf_counter() - t0
    secs, res = _oracle_step(o, "ratio", cfg["k"])
    return {"value": 1.0 / secs, "unit": "solves/s", "cores": cpu["usable_cores"], "kind": "port",
            "cpu": cpu,
            "sample": (f"one complete step of the oracle's lawlercpu restatement, OpenMP x{cpu['usable_cores']}: "
                       f"energies recomputed + rescale + in-edge sets + branch and bound, {secs:.1f}s "
                       f"({o.last_stats()['sweeps']} sweeps); the product graph, built once before "
                       f"({t_graph:.1f}s), is not counted, as the device keeps its layer template"),
            "result": {"objective": res[1], "cycle_edges": int(res[2].shape[0])}}


def _pair_config(workload, cfg, nodes_per_layer, layers, edges, world):
    """The `config` of a single-pair line, the same in both arms."""
    l2 = ("inputs larger than L2 (fp64 cost stream > 126 MB)" if 8 * edges >= L2_BYTES
          else "L2 flushed between timed steps (256 MB write; the cost streams are smaller than L2)")
    return {"workload": workload, "k": cfg["k"], "nodes_per_layer": int(nodes_per_layer), "layers": int(layers),
            "edges": int(edges), "cost_mode": [cfg["cost"], cfg["time"]], "parallelism": f"replicas x{world}",
            "l2": l2}


REFERENCE_BUDGET_S = 120.0  # timed CPU work of the reference arm's main configuration


def run_reference(args, workload, with_min_cost=False):
    """The oracle's lawlercpu on the host cores: after one untimed warm-up
    step, complete steps are timed until the budget is spent (at least one,
    at most --steps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    pair, cfg = _make_pair(workload, seed=args.seed)
    cpu = host_cpu()
    cores = cpu["usable_cores"]
    orc.set_threads(cores)
    o = _oracle_pair(orc, pair, cfg)
    o.generate()
    warm_s, _ = _oracle_step(o, "ratio", cfg["k"])
    n = max(1, min(args.steps, int(REFERENCE_BUDGET_S // max(warm_s, 1e-9))))
    samples, res = [], None
    for _ in range(n):
        secs, res = _oracle_step(o, "ratio", cfg["k"])
        samples.append(secs)
    mean_s = sum(samples) / len(samples)
    value = 1.0 / mean_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": n,
        "warmup": 1, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": 1000.0 * mean_s, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": _pair_config(workload, cfg, 3 * len(pair["EX"]) if cfg["conj"] else len(pair["VX"]),
                               len(pair["EY"]), o.product_space_rows(), int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port", "cpu": cpu,
                         "sample": (f"{n} complete steps of the oracle's lawlercpu restatement (energies "
                                    f"recomputed + rescale + in-edge sets + branch and bound), OpenMP x{cores}, "
                                    f"after one untimed warm-up step ({warm_s:.1f}s); steps timed until a "
                                    f"{REFERENCE_BUDGET_S:.0f}s budget, each {min(samples):.1f}-{max(samples):.1f}s")},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_s": samples, "result": {"objective": res[1], "cycle_edges": int(res[2].shape[0])},
    }
    if with_min_cost:
        secs, mres = _oracle_step(o, "min_cost", cfg["k"])
        line["dijkstracpu"] = {"value": 1.0 / secs, "unit": "solves/s", "steps": 1, "ms_per_step": 1000.0 * secs,
                               "sample": "one complete dijkstracpu step (energies recomputed + solve), "
                                         f"OpenMP x{cores}",
                               "result": {"objective": mres[1], "cycle_edges": int(mres[2].shape[0])}}
    return line


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
            "parallelism": f"one persistent launch, a team of CTAs per pair, replicas x{world}",
            "l2": "inputs larger than L2 (all pairs' cost streams together)"}


def _fwdbwd_config(workload, pairs, k, world):
    """The `config` of a fwd/bwd line, the same in both arms."""
    return {"workload": workload, "pairs": int(pairs), "vx": FWDBWD[workload][1], "vy": FWDBWD[workload][2],
            "k": int(k), "feature_dim": FWDBWD[workload][4],
            "parallelism": f"one persistent launch, a team of CTAs per pair, replicas x{world}",
            "l2": "per-pair streams of all pairs exceed L2"}


def _batch_pairs(name, seed, limit=0):
    """The batch's seeded pairs, built in parallel host processes (spawned, before any GPU work)."""
    import multiprocessing as mp

    specs = _batch_specs(name, seed)
    if limit > 0:
        specs = specs[:limit]  # the batch's first pairs (small profiling cases)
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        pairs = pool.map(_batch_pair, specs, chunksize=4)
    return specs, pairs


def run_batch(args, world, rank):
    """Batched serving: every step solves all pairs of the batch concurrently
    (solve_batch: costs regenerated and rescaled on the device, then one
    persistent launch in which teams of CTAs run each pair's whole ratio
    solve, largest pairs first).  Also timed: the same pairs solved one after
    the other with full-GPU teams (the plain per-pair GPU Lawler)."""
    specs, pairs = _batch_pairs(args.workload, args.seed + rank, args.pairs)
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
    launches = 0
    profiles = []
    with ClockSampler(dev) as clocks:
        for i in range(args.steps):
            torch.cuda.synchronize()
            n0 = cpg.kernel_launches()
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
            torch.cuda.synchronize()
            launches += cpg.kernel_launches() - n0
            profiles.append(cpg.last_batch_profile())
            for g, info, sp in zip(gens, infos, specs):
                bytes_moved += algorithmic_bytes_per_sweep(info, sp["k"], True) * g.last_stats()["sweeps"]
    pair_device_ms = sum(g.last_stats()["device_us"] for g in gens) / 1000.0
    # Bellman-Ford steps of the last step's solves, and where the lead thread's cycles went
    profs = [g.last_profile() for g in gens]
    bf_steps = sum(pr["steps"] for pr in profs)
    cycle_split = {k: sum(pr[k] for pr in profs) for k in ("cycles_relax", "cycles_handoff", "cycles_bookkeeping",
                                                           "cycles_sweep_tail", "cycles_stage_wait")}
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
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": f"{peak_kind} hbm_gbs", "kernel": "bf_batch_kernel (all pairs)",
                     "note": "algorithmic bytes of every sweep of every pair / batch step time"},
        "batch_profile": dict(_median_profile(profiles, pair_device_ms), bf_steps=bf_steps,
                              team_us_per_step=1000.0 * pair_device_ms / max(1, bf_steps),
                              lead_cycles_per_step={k: v / max(1, bf_steps) for k, v in cycle_split.items()}),
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = _batch_cpu_sample(specs, pairs)
    return line


def _median_profile(profiles, pair_device_ms):
    """The timed steps' batch phases (host wall clock, ms; medians over the
    steps) and the last step's summed per-pair device time: the team clock
    of each pair's whole ratio solve inside the persistent launch."""
    out = {k: statistics.median(p[k] for p in profiles) for k in profiles[0]} if profiles else {}
    out["pair_device_ms_sum"] = pair_device_ms
    return out


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
        # the pairs share their shapes: one batched distance computation (and
        # one backward) for all of them, the same per-pair values
        fds = torch.cdist(torch.stack(fX), torch.stack(fY)).double().unbind(0)
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
    launches = 0
    profiles = []
    with ClockSampler(dev) as clocks:
        for i in range(args.steps):
            torch.cuda.synchronize()
            n0 = cpg.kernel_launches()
            ev[i][0].record(stream)
            lam = step()
            ev[i][1].record(stream)
            torch.cuda.synchronize()
            launches += cpg.kernel_launches() - n0  # the library's kernels; torch's cdist/sum are not counted
            profiles.append(cpg.last_batch_profile())
    pair_device_ms = sum(g.last_stats()["device_us"] for g in gens) / 1000.0
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
    lam_e = ratio_cycle_objectives(fresh, torch.cdist(torch.stack(ax), torch.stack(by)).double().unbind(0), k)
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
        "gpu_launches": launches,
        "batch_profile": _median_profile(profiles, pair_device_ms),
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


SUB_CONFIGS = ("batch_256_plain_1k8k", "fwdbwd_32_plain_2k_100_k2", "conj_prune_20k_500_k4")


def _sub_args(args, workload, steps, warmup):
    import argparse

    sub = argparse.Namespace(**vars(args))
    sub.workload, sub.steps, sub.warmup = workload, steps, warmup
    return sub


def full_metric_line(args, world, rank):
    """The default line: the single-pair configuration at the top level, with
    its dijkstragpu timing and the CPU baseline, and the batched, fwd/bwd and
    large-pair configurations under "configs"."""
    import torch

    import cyclic_product_graphs as cpg

    # Every GPU timing first, the CPU baselines after them: host-driven steps
    # measured after the oracle's OpenMP runs (16 threads) were slower than
    # alone (fwd/bwd: 49 vs 21 ms per step), so the CPU work waits.
    line = measure_pair(args, world, rank, DEFAULT_WORKLOAD, args.steps, args.warmup, args.e2e_steps,
                        with_min_cost=True, with_cpu=False)
    sub_steps, sub_warmup = max(1, min(args.steps, args.sub_steps)), max(3, min(args.warmup, 3))
    configs = {}
    for name in SUB_CONFIGS:
        sub = _sub_args(args, name, sub_steps, sub_warmup)
        sub.no_cpu_baseline = True
        if name in BATCHES:
            configs[name] = run_batch(sub, world, rank)
        elif name in FWDBWD:
            configs[name] = run_fwdbwd(sub, world, rank)
        else:
            configs[name] = measure_pair(sub, world, rank, name, sub_steps, sub_warmup, 2)
        for key in ("metric", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "data"):
            configs[name].pop(key, None)
        torch.cuda.synchronize()
        gc.collect()
        cpg.release_cached_memory()
    line["configs"] = configs
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        pair, cfg = _make_pair(DEFAULT_WORKLOAD, seed=args.seed + rank)
        line["cpu_baseline"] = cpu_baseline(pair, cfg)
        for name in SUB_CONFIGS:
            if name in BATCHES:
                specs, pairs = _batch_pairs(name, args.seed + rank)
                configs[name]["cpu_baseline"] = _batch_cpu_sample(specs, pairs)
    return line


def full_reference_line(args):
    """The reference arm of the default line: complete lawlercpu steps of the
    single-pair configuration, one dijkstracpu step, and CPU samples of the
    batched and fwd/bwd configurations."""
    line = run_reference(args, DEFAULT_WORKLOAD, with_min_cost=True)
    configs = {}
    for name in SUB_CONFIGS:
        sub = _sub_args(args, name, 2, 1)
        if name in BATCHES:
            configs[name] = run_reference_batch(sub)
        elif name in FWDBWD:
            configs[name] = run_reference_fwdbwd(sub)
        else:
            configs[name] = {"impl": "reference", "unavailable": (
                "not timed on the CPU within the bench's budget: the oracle builds and holds the full product "
                "graph (721 M edges; about 30 GB of host memory with its costs and in-edge sets) and spends "
                "minutes per solve")}
        for key in ("metric", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "data"):
            configs[name].pop(key, None)
    line["configs"] = configs
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + sorted(BATCHES) + sorted(FWDBWD), default=None,
                    help="measure one configuration alone (default: the whole metric)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--sub-steps", type=int, default=5, help="timed steps of each configuration under 'configs'")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--pairs", type=int, default=0,
                    help="batched workload: solve only its first N pairs (small profiling cases; 0 = all)")
    args = ap.parse_args()
    world, rank, local = _dist_env()

    if args.impl == "reference":
        if rank == 0:
            if args.workload is None:
                line = full_reference_line(args)
            elif args.workload in BATCHES:
                line = run_reference_batch(args)
            elif args.workload in FWDBWD:
                line = run_reference_fwdbwd(args)
            else:
                line = run_reference(args, args.workload)
            print(json.dumps(line), flush=True)
        return

    # 32 host work queues let the stream route of batched solves (one stream
    # per pair: minimum-cost batches, the plain per-pair comparison's teams)
    # run side by side; CUDA's default of 8 serialises them.  Read when CUDA
    # starts, so it is set before anything touches the device.
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload is None:
        line = full_metric_line(args, world, rank)
    elif args.workload in BATCHES:
        line = run_batch(args, world, rank)
    elif args.workload in FWDBWD:
        line = run_fwdbwd(args, world, rank)
    else:
        line = measure_pair(args, world, rank, args.workload, args.steps, args.warmup, args.e2e_steps,
                            with_min_cost=False, with_cpu=not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
