"""The autotuner (no counterpart in the reference): it times candidate
Bellman-Ford team shapes for a graph's shape bucket, applies the fastest and
caches it in a JSON file; a graph of the same bucket then takes the cached
shape.  Every shape gives the oracle's result."""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu


def _same(got, want):
    assert got[0] == want[0] and got[1] == want[1] and np.array_equal(got[2], want[2])


def _conj(cpg, oracle, seed):
    p = synthetic.make_pair(n_vertices=300, n_curve=10, feat_dim=8, seed=seed)
    args = (p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], True, False, False)
    g, o = cpg.product_graph_generator(*args), oracle.OracleGenerator(*args)
    for x in (g, o):
        x.set_normals(p["NX"], p["NY"])
        x.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
    return g, o


def test_autotune_picks_applies_and_caches(cpg, oracle, tmp_path):
    g, o = _conj(cpg, oracle, 21)
    want = o.solve_with_cost_time_ratio("lawlercpu", 3)
    cache = tmp_path / "team_shapes.json"
    shapes = [(0, 0), (4, 640), (8, 320)]
    e = cpg.autotune(g, 3, candidates=shapes, cache_path=str(cache))
    assert not e["cached"] and cache.exists()
    assert [(c["ctas"], c["threads_per_cta"]) for c in e["candidates"]] == shapes
    assert all(c["bf_ms"] > 0 for c in e["candidates"])
    assert e["bf_ms"] == min(c["bf_ms"] for c in e["candidates"])
    # the chosen shape is applied
    g.generate()
    _same(g.solve_with_cost_time_ratio("lawlergpu", 3), want)
    prof = g.last_profile()
    if e["ctas"]:
        assert prof["ctas"] == e["ctas"]
    if e["threads_per_cta"]:
        assert prof["threads"] == e["threads_per_cta"]
    # every candidate gives the same result
    for shape in shapes:
        g.set_team_shape(*shape)
        g.generate()
        _same(g.solve_with_cost_time_ratio("lawlergpu", 3), want)
    # another graph of the same bucket takes the cached shape without timing
    g2, _ = _conj(cpg, oracle, 22)
    e2 = cpg.autotune(g2, 3, cache_path=str(cache))
    assert e2["cached"] and e2["bucket"] == e["bucket"]
    assert (e2["ctas"], e2["threads_per_cta"]) == (e["ctas"], e["threads_per_cta"])


def test_team_shape_rejects_bad_sizes(cpg, oracle):
    g, _ = _conj(cpg, oracle, 21)
    with pytest.raises(cpg.PGCError):
        g.set_team_shape(2, 100)
    with pytest.raises(cpg.PGCError):
        g.set_team_shape(-1, 0)
