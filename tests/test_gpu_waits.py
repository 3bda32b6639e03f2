"""Device-side robustness of the Bellman-Ford launch, without a GPU fault.

* Bounded waits: with a short poll limit (PGC_BF_SPIN_LIMIT), one CTA of a
  multi-CTA team is made to wait in its step hand-off for a word that no code
  writes (PGC_BF_TEST_STALL_CTA).  That wait runs out, raises the error word,
  every other CTA stops at its next wait, and the solve returns
  PGC_ERR_TIMEOUT promptly.  The same handle then solves as the oracle does.
  Nothing traps or faults: the waits simply give up.
* Literal walks: PGC_BF_LITERAL_WALKS=1 decides every negative candidate by
  the reference's predecessor walk instead of the lap function.  The walks run
  side by side in bounded rounds (cycle finding on the predecessor function);
  the answers must still equal the oracle's, for one-CTA and multi-CTA teams,
  plain and conjugate graphs, both solvers.

The reference has neither: its waits are unbounded and its walks serial
(ctr_bnb_subroutine.cuh:42-49, cost_time_ratio_solver.cpp:461-488).
"""
import time

import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu

PGC_ERR_TIMEOUT = -7


def _both(cpg, oracle, p, conj=False, cost="vanilla", time_mode="nomode"):
    args = (p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False, False)
    g = cpg.product_graph_generator(*args)
    o = oracle.OracleGenerator(*args)
    if conj:
        g.set_normals(p["NX"], p["NY"])
        o.set_normals(p["NX"], p["NY"])
    g.set_cost_time_ratio_mode(cost, time_mode)
    o.set_cost_time_ratio_mode(cost, time_mode)
    return g, o


def _same(got, want):
    assert got[0] == want[0]
    assert got[1] == want[1], (got[1], want[1])
    assert got[2].shape == want[2].shape
    assert np.array_equal(got[2], want[2])


@pytest.mark.parametrize("stall_cta", [0, 5])
def test_wait_timeout_returns_status_and_handle_recovers(cpg, oracle, monkeypatch, stall_cta):
    p = synthetic.make_pair(icosphere_level=3, n_curve=20, feat_dim=16, seed=4)
    g, o = _both(cpg, oracle, p)
    monkeypatch.setenv("PGC_BF_BLOCKS", "8")
    monkeypatch.setenv("PGC_BF_SPIN_LIMIT", "20000")
    monkeypatch.setenv("PGC_BF_TEST_STALL_CTA", str(stall_cta))
    t0 = time.perf_counter()
    with pytest.raises(cpg.PGCError) as e:
        g.solve_with_cost_time_ratio("lawlergpu", 2)
    assert e.value.code == PGC_ERR_TIMEOUT
    assert "ran out" in str(e.value)
    assert time.perf_counter() - t0 < 10.0
    assert g.last_profile()["ctas"] == 8
    # the hook off, the same handle (and its multi-CTA team) solves correctly
    monkeypatch.delenv("PGC_BF_TEST_STALL_CTA")
    monkeypatch.delenv("PGC_BF_SPIN_LIMIT")
    g.generate()
    _same(g.solve_with_cost_time_ratio("lawlergpu", 2), o.solve_with_cost_time_ratio("lawlercpu", 2))
    _same(g.solve_with_minimum_cost("dijkstragpu", 2), o.solve_with_minimum_cost("dijkstracpu", 2))


def test_stall_hook_outside_the_team_changes_nothing(cpg, oracle, monkeypatch):
    """A stall hook naming no CTA of the team leaves every wait as it is."""
    p = synthetic.make_pair(icosphere_level=2, n_curve=12, feat_dim=8, seed=6)
    g, o = _both(cpg, oracle, p)
    monkeypatch.setenv("PGC_BF_BLOCKS", "4")
    monkeypatch.setenv("PGC_BF_TEST_STALL_CTA", "99")
    _same(g.solve_with_cost_time_ratio("lawlergpu", 2), o.solve_with_cost_time_ratio("lawlercpu", 2))


@pytest.mark.parametrize("blocks", ["0", "8"])
@pytest.mark.parametrize("K,ny,seed", [(1, 12, 1), (2, 11, 2), (3, 14, 3)])
def test_literal_walks_plain(cpg, oracle, monkeypatch, blocks, K, ny, seed):
    monkeypatch.setenv("PGC_BF_LITERAL_WALKS", "1")
    if blocks != "0":
        monkeypatch.setenv("PGC_BF_BLOCKS", blocks)
    p = synthetic.make_pair(icosphere_level=3, n_curve=ny, feat_dim=16, seed=seed)
    g, o = _both(cpg, oracle, p)
    _same(g.solve_with_cost_time_ratio("lawlergpu", K), o.solve_with_cost_time_ratio("lawlercpu", K))
    st = g.last_stats()
    assert st["fallback_walks"] > 0, st
    _same(g.solve_with_minimum_cost("dijkstragpu", K), o.solve_with_minimum_cost("dijkstracpu", K))


@pytest.mark.parametrize("blocks", ["0", "12"])
def test_literal_walks_conjugate(cpg, oracle, monkeypatch, blocks):
    monkeypatch.setenv("PGC_BF_LITERAL_WALKS", "1")
    if blocks != "0":
        monkeypatch.setenv("PGC_BF_BLOCKS", blocks)
    p = synthetic.make_pair(n_vertices=300, n_curve=10, feat_dim=8, seed=21)
    g, o = _both(cpg, oracle, p, conj=True, cost="vanilla", time_mode="lengthnormalisation")
    _same(g.solve_with_cost_time_ratio("lawlergpu", 3), o.solve_with_cost_time_ratio("lawlercpu", 3))
    assert g.last_stats()["fallback_walks"] > 0
