"""pgc_release_cached_memory returns the cached device and pinned host blocks;
handles created afterwards allocate afresh and solve the same."""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu


def test_release_cached_memory_between_handles(cpg):
    p = synthetic.make_pair(icosphere_level=2, n_curve=10, feat_dim=8, seed=6)
    args = (p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], False, False, False)
    g = cpg.product_graph_generator(*args)
    first = g.solve_with_cost_time_ratio("lawlergpu", 2)
    del g
    cpg.release_cached_memory()
    g = cpg.product_graph_generator(*args)
    again = g.solve_with_cost_time_ratio("lawlergpu", 2)
    assert first[0] == again[0] and first[1] == again[1] and np.array_equal(first[2], again[2])
    cpg.release_cached_memory()  # with a live handle: only free blocks go
    assert g.solve_with_minimum_cost("dijkstragpu", 2)[2].shape[1] == 4
