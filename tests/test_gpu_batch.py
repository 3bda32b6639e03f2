"""Batched solves (solve_batch / pgc_solve_batch): many graphs of uneven size
solved concurrently with one-CTA teams must return exactly what the oracle
returns for each of them, for the ratio and the minimum-cost solver, and a
failing member must be reported without affecting the others."""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu


def _same(got, want):
    assert got[0] == want[0]
    assert got[1] == want[1], (got[1], want[1])
    assert np.array_equal(got[2], want[2])


def _specs():
    # (n_vertices, n_curve, K, conjugate, seed); the seeds keep the oracle's
    # branch-and-bound short (some pairs need thousands of branches)
    return [(150, 10, 2, False, 10), (300, 14, 3, False, 11), (90, 8, 1, False, 12), (200, 12, 2, True, 14),
            (120, 6, 3, True, 14), (400, 16, 2, False, 15), (250, 9, 2, False, 16), (180, 10, 3, True, 13)]


def _build(cpg, oracle, spec):
    nv, m, K, conj, seed = spec
    p = synthetic.make_pair(n_vertices=nv, n_curve=m, feat_dim=16, seed=seed)
    args = (p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False, False)
    g, o = cpg.product_graph_generator(*args), oracle.OracleGenerator(*args)
    if conj:
        for x in (g, o):
            x.set_normals(p["NX"], p["NY"])
            x.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
    g.set_max_depth_cost_time_ratio(K)
    o.set_max_depth_cost_time_ratio(K)
    return g, o


@pytest.mark.parametrize("solver,ref", [("lawlergpu", "lawlercpu"), ("dijkstragpu", "dijkstracpu")])
def test_batch_matches_oracle(cpg, oracle, solver, ref):
    pairs = [_build(cpg, oracle, s) for s in _specs()]
    gens = [g for g, _ in pairs]
    got = cpg.solve_batch(gens, solver, None, ctas_per_graph=1, workers=4, regenerate=True)
    for (g, o), res in zip(pairs, got):
        want = o.solve_with_cost_time_ratio(ref) if solver.startswith("lawler") else o.solve_with_minimum_cost(ref)
        _same(res, want)
        assert g.last_profile()["ctas"] == 1


def test_batch_equals_single_solves_with_full_teams(cpg, oracle):
    pairs = [_build(cpg, oracle, s) for s in _specs()[:4]]
    batched = cpg.solve_batch([g for g, _ in pairs], "lawlergpu", None, ctas_per_graph=2)
    for (g, _), res in zip(pairs, batched):
        g.generate()
        _same(res, g.solve_with_cost_time_ratio("lawlergpu"))


def test_batch_reports_a_failing_member(cpg, oracle):
    good = [_build(cpg, oracle, s)[0] for s in _specs()[:3]]
    p = synthetic.make_pair(n_vertices=100, n_curve=8, feat_dim=8, seed=3)
    bad = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], True, False)  # no normals
    with pytest.raises(cpg.PGCError, match="graph 1 of the batch failed"):
        cpg.solve_batch([good[0], bad, good[1], good[2]], "lawlergpu", None)
    # the others were solved all the same
    _, o = _build(cpg, oracle, _specs()[2])
    _same(good[2]._result(), o.solve_with_cost_time_ratio("lawlercpu"))


def test_batch_rejects_repeated_generators(cpg, oracle):
    g, _ = _build(cpg, oracle, _specs()[0])
    with pytest.raises(ValueError):
        cpg.solve_batch([g, g], "lawlergpu", 2)
