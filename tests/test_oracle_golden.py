"""Pins the CPU oracle against exact known answers (tests/golden/toy_cases.json).

The fixtures come from tests/golden/make_golden.py, which builds the toy
product graphs, their costs and the rescale from their definitions and finds
the optima by exact enumeration -- independently of the oracle.
"""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "toy_cases.json")) as f:
    CASES = json.load(f)["cases"]


def _arrays(c):
    return (np.array(c["VX"]), np.array(c["EX"], dtype=np.int32), np.array(c["VY"]), np.array(c["EY"], dtype=np.int32),
            np.array(c["feat_diff"]))


def check_case(gen_factory, c):
    """Ratio solve, then min-cost on the rescaled costs, then min-cost on raw costs."""
    VX, EX, VY, EY, fd = _arrays(c)
    g = gen_factory(VX, EX, VY, EY, fd)
    g.set_cost_time_ratio_mode("vanilla", "nomode")
    passes, obj, m = g.solve_with_cost_time_ratio("lawlercpu", c["K"])
    want = Fraction(c["ratio"][0], c["ratio"][1])
    assert passes
    assert obj == np.float32(float(want)), (obj, float(want))
    edges = sorted(g.last_cycle_edges().tolist())
    assert edges in c["ratio_cycles"], "returned ratio cycle is not one of the optimal cycles"
    assert m.shape == (len(edges), 4)

    passes, obj, m = g.solve_with_minimum_cost("dijkstracpu", c["K"])
    assert passes
    assert obj == np.float32(c["min_cost_after_ratio"])
    assert sorted(g.last_cycle_edges().tolist()) in c["min_cost_after_ratio_cycles"]

    g2 = gen_factory(VX, EX, VY, EY, fd)
    passes, obj, m = g2.solve_with_minimum_cost("dijkstracpu", c["K"])
    want = Fraction(c["min_cost_raw"][0], c["min_cost_raw"][1])
    assert obj == np.float32(float(want))
    assert sorted(g2.last_cycle_edges().tolist()) in c["min_cost_raw_cycles"]


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_known_answers(oracle, c):
    check_case(lambda *a: oracle.OracleGenerator(*a, False, False), c)


def test_fixture_product_space_matches_oracle(oracle):
    """The fixture generator's product graph equals the oracle's restatement."""
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden

    c = CASES[0]
    VX, EX, VY, EY, fd = _arrays(c)
    ps, src, trgt = make_golden.plain_product(EX, EY, VX.shape[0])
    o = oracle.OracleGenerator(VX, EX, VY, EY, fd, False, False)
    assert np.array_equal(o.get_product_space(), ps)
    s2, t2 = o.get_src_trgt()
    assert np.array_equal(s2, np.array(src)) and np.array_equal(t2, np.array(trgt))
