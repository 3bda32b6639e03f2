"""Ratio solves whose Lawler cycle wraps more than once, so that the branch
and bound splits the layer-0 start nodes into branches
(cost_time_ratio_solver.cpp:611-634, :804-851; branch, :142-179).

The cases are small plain and conjugate graphs, pruned or not, K 1-3, with
integer edge costs drawn at random (set_cost_vector): such costs often make
the optimum wrap, where the synthetic energies rarely do.  The oracle
branches on each (branches > 1); the device must branch the same number of
times and return the same answer, as a single solve and inside a batch,
where the batched device solve hands such graphs back to the host.
"""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu

# (seed, icosphere level, curve points, K, conjugate, pruned, largest cost):
# the seed draws all the others, then the costs
CASES = [(162, 1, 3, 3, False, False, 100), (290, 0, 5, 2, False, False, 10), (150, 1, 3, 2, True, False, 1000),
         (326, 0, 3, 3, True, False, 1000), (287, 1, 8, 2, True, True, 3), (84, 1, 7, 1, True, True, 100),
         (155, 0, 4, 3, True, True, 10), (216, 1, 8, 1, True, False, 10), (38, 0, 5, 1, False, False, 100),
         (120, 0, 8, 1, False, True, 10), (282, 1, 6, 2, False, True, 100)]


def _draw(seed):
    rng = np.random.default_rng(seed)
    shape = (int(rng.integers(0, 2)), int(rng.integers(3, 9)), int(rng.integers(1, 4)), bool(rng.integers(0, 2)),
             bool(rng.integers(0, 2)), int(rng.choice([3, 10, 100, 1000])))
    return rng, shape


def _make(factory, case):
    seed, level, ny, K, conj, prune, hi = case
    p = synthetic.make_pair(icosphere_level=level, n_curve=ny, feat_dim=4, seed=seed)
    g = factory(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False, prune)
    if conj:
        g.set_normals(p["NX"], p["NY"])
        g.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
    return g


def _pair(cpg, oracle, case):
    rng, shape = _draw(case[0])
    assert shape == tuple(case[1:])
    g = _make(cpg.product_graph_generator, case)
    o = _make(oracle.OracleGenerator, case)
    rows, cols = o.get_cost_vector().shape
    c = rng.integers(1, case[6] + 1, size=(rows, cols)).astype(np.float64)
    g.set_cost_vector(c)
    o.set_cost_vector(c)
    g.set_max_depth_cost_time_ratio(case[3])
    o.set_max_depth_cost_time_ratio(case[3])
    return g, o


def _same(got, want):
    assert got[0] == want[0]
    assert got[1] == want[1], (got[1], want[1])
    assert np.array_equal(got[2], want[2])


@pytest.mark.parametrize("case", CASES, ids=[f"s{c[0]}" for c in CASES])
def test_ratio_solve_branches_like_the_oracle(cpg, oracle, case):
    g, o = _pair(cpg, oracle, case)
    want = o.solve_with_cost_time_ratio("lawlercpu")
    assert o.last_stats()["branches"] > 1  # the case does branch
    _same(g.solve_with_cost_time_ratio("lawlergpu"), want)
    assert g.last_stats()["branches"] == o.last_stats()["branches"]


def test_branching_graphs_in_a_batch(cpg, oracle):
    pairs = [_pair(cpg, oracle, c) for c in CASES]
    got = cpg.solve_batch([g for g, _ in pairs], "lawlergpu", None)
    for (g, o), res in zip(pairs, got):
        _same(res, o.solve_with_cost_time_ratio("lawlercpu"))
        assert g.last_stats()["branches"] == o.last_stats()["branches"]
