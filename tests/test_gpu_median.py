"""The ratio solve's in-place rescale (cost_time_ratio_solver.cpp:709-721 with
utils::median, utils.hpp:196-209) on cost columns chosen to reach every path
of the device's radix selection: every value equal (all 64 key bits fixed),
a few values repeated many times, an even count whose two middle values lie
in different top digits (the second one is the smallest key above the
selected bucket), negative values, a median below 0.001 (the factor's
floor), and a typical spread.  Both columns are set (cost and time), so both
selections run; after the solve the device's rescaled columns, objective
and matching must equal the oracle's bit for bit.
"""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu


def _column(kind, rows, rng):
    if kind == "equal":
        return np.full(rows, 3.25)
    if kind == "few":
        return rng.choice([0.5, 7.0, 19.0], size=rows, p=[0.3, 0.45, 0.25])
    if kind == "split":
        # even count, half 1.0 and half 2.0: the middle pair straddles two top digits
        c = np.full(rows, 2.0)
        c[: rows // 2] = 1.0
        return rng.permutation(c)
    if kind == "signed":
        return rng.normal(size=rows) * 5.0
    if kind == "tiny":
        return np.abs(rng.normal(size=rows)) * 1e-5 + 1e-7
    return np.abs(rng.normal(size=rows)) * 40.0 + 1.0


KINDS = ["equal", "few", "split", "signed", "tiny", "spread"]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("conj,odd,large", [(False, False, False), (True, False, False), (False, True, False),
                                            (False, False, True)])
def test_rescale_selection_paths_match_oracle(cpg, oracle, kind, conj, odd, large):
    # an icosphere with six curve points gives an even count of costs (the
    # median is the mean of the two middle values); a 101-vertex mesh with five
    # curve points an odd one; a 2,000-vertex mesh with 40 curve points over
    # half a million, so that columns of few distinct values need every digit
    # pass (their buckets stay above the compaction's 65,536 values)
    if large:
        p = synthetic.make_pair(n_vertices=2000, n_curve=40, feat_dim=4, seed=31)
    elif odd:
        p = synthetic.make_pair(n_vertices=101, n_curve=5, feat_dim=4, seed=31)
    else:
        p = synthetic.make_pair(icosphere_level=1, n_curve=6, feat_dim=4, seed=31)
    args = (p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False, False)
    g, o = cpg.product_graph_generator(*args), oracle.OracleGenerator(*args)
    if conj:
        for x in (g, o):
            x.set_normals(p["NX"], p["NY"])
    rows = o.get_cost_vector().shape[0]
    assert rows % 2 == (1 if odd else 0)
    assert not large or rows > 4 * 65536
    rng = np.random.default_rng(KINDS.index(kind))
    cost = _column(kind, rows, rng)
    time = _column("spread" if kind == "equal" else kind, rows, rng)
    if kind == "signed":
        time = np.abs(time) + 0.5  # times stay positive, as the energies' are
    c = np.stack([cost, time], axis=1)
    g.set_cost_vector(c)
    o.set_cost_vector(c)
    try:
        want = o.solve_with_cost_time_ratio("lawlercpu", 2)
    except RuntimeError as e:  # the reference's "no nodes in branch" end: the device must stop the same way
        with pytest.raises(cpg.PGCError, match=str(e)):
            g.solve_with_cost_time_ratio("lawlergpu", 2)
        assert np.array_equal(g.get_cost_vector(), o.get_cost_vector())
        return
    got = g.solve_with_cost_time_ratio("lawlergpu", 2)
    assert np.array_equal(g.get_cost_vector(), o.get_cost_vector())
    assert got[0] == want[0]
    assert got[1] == want[1] or (np.isnan(got[1]) and np.isnan(want[1]))
    assert np.array_equal(got[2], want[2])
