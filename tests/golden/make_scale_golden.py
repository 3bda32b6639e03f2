"""Generates tests/golden/scale_cases.json: the oracle's answers on benchmark
configurations at their stated sizes.

The cases (tests/scale_inputs.py) are the single-pair GPU configuration
(conjugate, 5,000-vertex mesh x 200-point curve, K = 3), four pairs of the
differentiation configuration (plain, 2,000 x 100, K = 2) and eight pairs of
the batched-serving configuration spanning its size distribution.  For each,
the oracle -- the CPU restatement of the reference solvers, run on one
thread, since the reference's cycle choice races between OpenMP threads --
solves with lawlercpu and dijkstracpu on fresh generators.  The fixture
records the input digest, both objectives, the matchings and the oracle's
counters.

Run from the repository root:

    python tests/golden/make_scale_golden.py [--jobs N] [--only NAME ...]

Cases run in parallel processes (one oracle thread each); an existing
fixture file is updated case by case.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "scale_cases.json")


def _paths():
    for p in (os.path.join(ROOT, "product-graph-cycles_b200"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)


def solve_case(case):
    _paths()
    import oracle as orc
    import scale_inputs as si

    orc.set_threads(1)
    t0 = time.time()
    pair = si.make_inputs(case)
    res = si.oracle_results(orc, case, pair)
    return case["name"], {"case": case, "digest": si.input_digest(pair), "results": res,
                          "oracle_seconds": round(time.time() - t0, 1)}


def main():
    _paths()
    import scale_inputs as si

    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=max(1, (os.cpu_count() or 2) - 1))
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args()
    cases = [c for c in si.CASES if not args.only or c["name"] in args.only]
    data = {"cases": {}}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    # the largest first, so the pool's tail is short
    cases.sort(key=lambda c: -(c["n_vertices"] * c["n_curve"] * (6 if c["conj"] else 1)))
    with mp.get_context("spawn").Pool(args.jobs) as pool:
        for name, entry in pool.imap_unordered(solve_case, cases):
            data["cases"][name] = entry
            data["cases"] = dict(sorted(data["cases"].items()))
            with open(OUT + ".tmp", "w") as f:
                json.dump(data, f, separators=(",", ":"))
            os.replace(OUT + ".tmp", OUT)
            print(f"{name}: {entry['oracle_seconds']}s", flush=True)


if __name__ == "__main__":
    main()
