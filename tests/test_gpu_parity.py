"""GPU parity: the sm_100a solvers against the CPU oracle on identical seeded inputs.

Matchings must be bit-identical and objectives equal; cost vectors of
arithmetic-only modes must be bit-identical, those involving SO(3) distances
(acos/pow) agree to a relative 1e-9 and the solvers are then compared on the
same cost vector.
"""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu


def _pair(level=None, nv=200, ny=12, dim=16, seed=0):
    return synthetic.make_pair(icosphere_level=level, n_vertices=nv, n_curve=ny, feat_dim=dim, seed=seed)


def _both(cpg, oracle, p, conj=False, reg=False, prune=False, cost="vanilla", time="nomode", normals=None):
    args = (p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, reg, prune)
    g = cpg.product_graph_generator(*args)
    o = oracle.OracleGenerator(*args)
    if conj or normals:
        g.set_normals(p["NX"], p["NY"])
        o.set_normals(p["NX"], p["NY"])
    g.set_cost_time_ratio_mode(cost, time)
    o.set_cost_time_ratio_mode(cost, time)
    return g, o


def _same(got, want):
    assert got[0] == want[0]
    assert got[1] == want[1], (got[1], want[1])
    assert got[2].shape == want[2].shape, (got[2].shape, want[2].shape)
    assert np.array_equal(got[2], want[2])


@pytest.mark.parametrize("K", [1, 2, 3])
@pytest.mark.parametrize("ny", [12, 11])
def test_plain_ratio_and_min_cost(cpg, oracle, K, ny):
    p = _pair(level=2, ny=ny, seed=K + ny)
    g, o = _both(cpg, oracle, p)
    assert np.array_equal(g.get_product_space(), o.get_product_space())
    assert np.array_equal(g.get_cost_vector(), o.get_cost_vector())
    _same(g.solve_with_cost_time_ratio("lawlergpu", K), o.solve_with_cost_time_ratio("lawlercpu", K))
    assert np.array_equal(g.get_cost_vector(), o.get_cost_vector())  # rescaled in place on both
    _same(g.solve_with_minimum_cost("dijkstragpu", K), o.solve_with_minimum_cost("dijkstracpu", K))


def test_plain_min_cost_unscaled(cpg, oracle):
    p = _pair(level=2, ny=10, seed=5)
    g, o = _both(cpg, oracle, p)
    _same(g.solve_with_minimum_cost("dijkstragpu", 2), o.solve_with_minimum_cost("dijkstracpu", 2))


@pytest.mark.parametrize("reg,cost,time", [(True, "vanilla", "nomode"), (False, "feature", "lengthnormalisation"),
                                           (True, "feature", "lengthnormalisation")])
def test_plain_modes(cpg, oracle, reg, cost, time):
    p = _pair(level=2, ny=14, seed=7)
    g, o = _both(cpg, oracle, p, reg=reg, cost=cost, time=time)
    assert np.array_equal(g.get_cost_vector(), o.get_cost_vector())
    _same(g.solve_with_cost_time_ratio("lawlergpu", 2), o.solve_with_cost_time_ratio("lawlercpu", 2))
    _same(g.solve_with_minimum_cost("dijkstragpu", 2), o.solve_with_minimum_cost("dijkstracpu", 2))


def test_plain_prune(cpg, oracle):
    p = _pair(level=2, ny=12, seed=9)
    g, o = _both(cpg, oracle, p, prune=True)
    assert np.array_equal(g.get_product_space(), o.get_product_space())
    _same(g.solve_with_cost_time_ratio("lawlergpu", 2), o.solve_with_cost_time_ratio("lawlercpu", 2))
    _same(g.solve_with_minimum_cost("dijkstragpu", 2), o.solve_with_minimum_cost("dijkstracpu", 2))


def test_two_layers(cpg, oracle):
    p = _pair(level=1, ny=2, seed=11)
    g, o = _both(cpg, oracle, p)
    _same(g.solve_with_cost_time_ratio("lawlergpu", 2), o.solve_with_cost_time_ratio("lawlercpu", 2))
    _same(g.solve_with_minimum_cost("dijkstragpu", 2), o.solve_with_minimum_cost("dijkstracpu", 2))


@pytest.mark.parametrize("cost,time,prune", [("vanilla", "lengthnormalisation", False), ("vanilla", "", False),
                                             ("vanilla", "vanilla", False), ("vanilla", "lengthnormalisation", True)])
def test_conjugate_arithmetic_modes(cpg, oracle, cost, time, prune):
    p = _pair(level=1, ny=8, dim=8, seed=13)
    g, o = _both(cpg, oracle, p, conj=True, prune=prune, cost=cost, time=time)
    assert np.array_equal(g.get_product_space(), o.get_product_space())
    assert np.array_equal(g.get_cost_vector(), o.get_cost_vector())
    _same(g.solve_with_cost_time_ratio("lawlergpu", 2), o.solve_with_cost_time_ratio("lawlercpu", 2))
    _same(g.solve_with_minimum_cost("dijkstragpu", 2), o.solve_with_minimum_cost("dijkstracpu", 2))


@pytest.mark.parametrize("cost,time,prune", [("vanilla", "vanilla", False), ("feature", "plainso3", False),
                                             ("feature", "robustso3", False), ("robustso3", "feature", False),
                                             ("plainso3", "feature", False), ("robustso3", "feature", True),
                                             ("feature", "plainso3", True)])
def test_conjugate_so3_modes(cpg, oracle, cost, time, prune):
    p = _pair(level=1, ny=8, dim=8, seed=17)
    g, o = _both(cpg, oracle, p, conj=True, reg=True, prune=prune, cost=cost, time=time)
    eg, eo = g.get_cost_vector(), o.get_cost_vector()
    assert eg.shape == eo.shape
    np.testing.assert_allclose(eg, eo, rtol=1e-9, atol=1e-9)
    o.set_cost_vector(eg)  # same costs on both sides from here on
    # a pruned graph can leave the ratio solver's first branch empty; the
    # reference then stops with "no nodes in branch", and so must the device
    _same_or_same_error(lambda: g.solve_with_cost_time_ratio("lawlergpu", 2),
                        lambda: o.solve_with_cost_time_ratio("lawlercpu", 2))
    _same(g.solve_with_minimum_cost("dijkstragpu", 2), o.solve_with_minimum_cost("dijkstracpu", 2))


def _same_or_same_error(device, ref):
    try:
        want = ref()
    except Exception as e:  # the oracle's error: the device must raise the same message
        msg = str(e)
        assert msg
        with pytest.raises(Exception, match=msg):
            device()
        return
    _same(device(), want)


def test_config0_shape(cpg, oracle):
    """Plain method, 642-vertex icosphere, 60-point curve, k=2, vanilla / nomode."""
    p = synthetic.make_pair(icosphere_level=3, n_curve=60, feat_dim=32, seed=0)
    g, o = _both(cpg, oracle, p)
    _same(g.solve_with_cost_time_ratio("lawlergpu", 2), o.solve_with_cost_time_ratio("lawlercpu", 2))
    _same(g.solve_with_minimum_cost("dijkstragpu", 2), o.solve_with_minimum_cost("dijkstracpu", 2))


def test_multi_cta_team(cpg, oracle, monkeypatch):
    """The cooperative multi-CTA Bellman-Ford launch gives the same answers."""
    monkeypatch.setenv("PGC_BF_BLOCKS", "8")
    p = synthetic.make_pair(icosphere_level=3, n_curve=20, feat_dim=16, seed=2)
    g, o = _both(cpg, oracle, p)
    _same(g.solve_with_cost_time_ratio("lawlergpu", 3), o.solve_with_cost_time_ratio("lawlercpu", 3))
    _same(g.solve_with_minimum_cost("dijkstragpu", 3), o.solve_with_minimum_cost("dijkstracpu", 3))


@pytest.mark.parametrize("stage", ["2", "0"])
def test_staging_modes(cpg, oracle, monkeypatch, stage):
    """Source indices staged alone (costs and times read in place after an
    L2 prefetch), and no staging at all, on a multi-CTA conjugate team."""
    monkeypatch.setenv("PGC_BF_BLOCKS", "12")
    monkeypatch.setenv("PGC_BF_STAGE_SRC", stage)
    if stage == "0":
        monkeypatch.setenv("PGC_BF_STAGE", "0")
    p = _pair(nv=300, ny=10, dim=8, seed=21)
    g, o = _both(cpg, oracle, p, conj=True, cost="vanilla", time="lengthnormalisation")
    _same(g.solve_with_cost_time_ratio("lawlergpu", 3), o.solve_with_cost_time_ratio("lawlercpu", 3))
    _same(g.solve_with_minimum_cost("dijkstragpu", 3), o.solve_with_minimum_cost("dijkstracpu", 3))


def test_conjugate_multi_cta(cpg, oracle, monkeypatch):
    monkeypatch.setenv("PGC_BF_BLOCKS", "16")
    p = _pair(nv=300, ny=10, dim=8, seed=21)
    g, o = _both(cpg, oracle, p, conj=True, cost="vanilla", time="lengthnormalisation")
    _same(g.solve_with_cost_time_ratio("lawlergpu", 3), o.solve_with_cost_time_ratio("lawlercpu", 3))
    _same(g.solve_with_minimum_cost("dijkstragpu", 3), o.solve_with_minimum_cost("dijkstracpu", 3))
