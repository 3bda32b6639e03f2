"""Inputs of the full-size parity cases (tests/golden/scale_cases.json).

Each case is one shape pair of a benchmark configuration at its stated size,
drawn by the seeded synthetic generator.  The fixture records a SHA-256
digest of the inputs, so a test can tell whether the pair it regenerates is
the one the fixture was solved on.
"""
from __future__ import annotations

import hashlib

import numpy as np

from cyclic_product_graphs import synthetic

# The single-pair GPU configuration: conjugate graph of a 5,000-vertex mesh
# and a 200-point curve, 64-d features, K = 3, ("vanilla",
# "lengthnormalisation"); seed 1, the benchmark's pair.
CFG1 = dict(name="cfg1_conj_5k_200_k3_s1", n_vertices=5000, n_curve=200, feat_dim=64, seed=1, conj=True,
            prune=False, cost="vanilla", time="lengthnormalisation", k=3)

# The differentiation configuration: plain graphs, |VX| = 2,000, |VY| = 100,
# K = 2, 64-d features; four of its 32 pairs (the benchmark's seeds 100000+i).
CFG3 = [dict(name=f"cfg3_plain_2k_100_k2_s{100000 + i}", n_vertices=2000, n_curve=100, feat_dim=64,
             seed=100000 + i, conj=False, prune=False, cost="vanilla", time="nomode", k=2) for i in range(4)]


def _cfg2_sample(count=8, seed=1):
    """Eight pairs of the batched-serving configuration (|VX| ~ U[1k, 8k],
    |VY| ~ U[50, 250] even, K in {2, 3}, 32-d features), drawn as the
    benchmark draws its 256 and picked at evenly spaced ranks of their size
    |VX| x |VY|, so the sample spans the distribution."""
    rng = np.random.default_rng(seed)
    specs = [dict(nv=int(rng.integers(1000, 8001)), m=2 * int(rng.integers(25, 126)), k=int(rng.choice((2, 3))),
                  seed=seed * 100000 + i) for i in range(256)]
    order = sorted(range(len(specs)), key=lambda i: (specs[i]["nv"] * specs[i]["m"], i))
    picks = [order[round(j * (len(order) - 1) / (count - 1))] for j in range(count)]
    return [dict(name=f"cfg2_plain_{specs[i]['nv']}_{specs[i]['m']}_k{specs[i]['k']}_s{specs[i]['seed']}",
                 n_vertices=specs[i]["nv"], n_curve=specs[i]["m"], feat_dim=32, seed=specs[i]["seed"], conj=False,
                 prune=False, cost="vanilla", time="nomode", k=specs[i]["k"]) for i in picks]


CFG2 = _cfg2_sample()
CASES = [CFG1] + CFG3 + CFG2


def make_inputs(case):
    """The case's pair: VX, EX, VY, EY, feat_diff (and NX, NY for conjugate graphs)."""
    p = synthetic.make_pair(n_vertices=case["n_vertices"], n_curve=case["n_curve"], feat_dim=case["feat_dim"],
                            seed=case["seed"], with_normals=case["conj"])
    keys = ("VX", "EX", "VY", "EY", "feat_diff") + (("NX", "NY") if case["conj"] else ())
    return {k: p[k] for k in keys}


def input_digest(pair):
    """SHA-256 over the input arrays' shapes, dtypes and bytes, in a fixed order."""
    h = hashlib.sha256()
    for k in ("VX", "EX", "VY", "EY", "feat_diff", "NX", "NY"):
        if k in pair:
            a = np.ascontiguousarray(pair[k])
            h.update(f"{k}:{a.dtype.str}:{a.shape}".encode())
            h.update(a.tobytes())
    return h.hexdigest()


def generator(factory, case, pair):
    """A generator (the product's or the oracle's) for the case's pair, its normals and modes set."""
    g = factory(pair["VX"], pair["EX"], pair["VY"], pair["EY"], pair["feat_diff"], case["conj"], False,
                case["prune"])
    if case["conj"]:
        g.set_normals(pair["NX"], pair["NY"])
    g.set_cost_time_ratio_mode(case["cost"], case["time"])
    return g


def oracle_results(orc, case, pair):
    """The oracle's lawlercpu and dijkstracpu answers (one thread: the
    reference's cycle choice races between OpenMP threads), each on a fresh
    generator, as {"ratio": ..., "min_cost": ...}."""
    out = {}
    for solver in ("ratio", "min_cost"):
        o = generator(orc.OracleGenerator, case, pair)
        r = o.solve_with_cost_time_ratio("lawlercpu", case["k"]) if solver == "ratio" else \
            o.solve_with_minimum_cost("dijkstracpu", case["k"])
        out[solver] = {"passes": bool(r[0]), "objective": float(r[1]), "matching": r[2].tolist(),
                       "edges": o.last_cycle_edges().tolist(), "stats": o.last_stats()}
        del o
    return out
