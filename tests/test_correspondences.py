"""vertex_correspondences: the matching-to-correspondence step of the
reference's usage example (README.md:79-85), on matchings from the oracle's
solvers (plain and conjugate) and on malformed input.  No GPU: the helper is
host-side column selection."""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic


def _solve(oracle, conj, ratio):
    p = synthetic.make_pair(n_vertices=60, n_curve=8, feat_dim=4, seed=1)
    g = oracle.OracleGenerator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False)
    if conj:
        g.set_normals(p["NX"], p["NY"])
    g.set_cost_time_ratio_mode("vanilla", "lengthnormalisation" if conj else "nomode")
    r = g.solve_with_cost_time_ratio("lawlercpu", 2) if ratio else g.solve_with_minimum_cost("dijkstracpu", 2)
    return p, r


@pytest.mark.parametrize("conj", [False, True])
@pytest.mark.parametrize("ratio", [True, False])
def test_correspondences_follow_the_cycle(cpg, oracle, conj, ratio):
    p, (passes, _, m) = _solve(oracle, conj, ratio)
    assert passes
    c = cpg.vertex_correspondences(m)
    assert c.dtype == np.int32 and c.shape == (len(m), 2)
    # the README's selection
    assert np.array_equal(c[:, 0], m[:, 3 if conj else 2]) and np.array_equal(c[:, 1], m[:, 0])
    assert np.array_equal(cpg.vertex_correspondences(m, conjugate=conj), c)
    # each row ends where the next starts, around the cycle
    w = 3 if conj else 2
    nxt = np.roll(m, -1, axis=0)
    assert np.array_equal(m[:, 1:w], nxt[:, :w - 1]) and np.array_equal(m[:, w + 1:], nxt[:, w:2 * w - 1])
    # a cycle that passes every layer once visits every curve vertex and stays on shape X
    assert set(c[:, 1].tolist()) == set(range(len(p["VY"])))
    assert c[:, 0].min() >= 0 and c[:, 0].max() < len(p["VX"])


def test_correspondences_reject_malformed_matchings(cpg):
    with pytest.raises(ValueError):
        cpg.vertex_correspondences(np.zeros((3, 5), np.int32))
    with pytest.raises(ValueError):
        cpg.vertex_correspondences(np.zeros(4, np.int32))
    with pytest.raises(ValueError):
        cpg.vertex_correspondences(np.zeros((3, 4), np.int32), conjugate=True)
    assert cpg.vertex_correspondences(np.zeros((0, 6), np.int32)).shape == (0, 2)
