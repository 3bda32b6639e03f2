"""The "export" solver writes the reference's replay files (VX, VY, EX, EY,
FeatDiffMatrix, NX, NY as CSV, product_graph_generators.cpp:272-282);
load_export reads them back exactly and from_export replays the problem with
the same result."""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("conj", [False, True])
def test_export_round_trip_replays_the_solve(cpg, tmp_path, monkeypatch, conj):
    p = synthetic.make_pair(icosphere_level=2, n_curve=8, feat_dim=8, seed=4)
    monkeypatch.chdir(tmp_path)
    g = cpg.product_graph_generator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False, False)
    if conj:
        g.set_normals(p["NX"], p["NY"])
        g.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
    passes, obj, matching = g.solve_with_cost_time_ratio("export")
    assert (passes, obj, matching.shape) == (False, -1.0, (4, 1))  # the reference's export tuple
    d = cpg.load_export(str(tmp_path))
    for key, want in (("VX", p["VX"]), ("VY", p["VY"]), ("EX", p["EX"]), ("EY", p["EY"]), ("feat_diff", p["feat_diff"])):
        assert np.array_equal(d[key], want), key
    assert ("NX" in d) == conj
    if conj:
        assert np.array_equal(d["NX"], p["NX"]) and np.array_equal(d["NY"], p["NY"])
    r = cpg.from_export(str(tmp_path), conj, False, False)
    if conj:
        r.set_cost_time_ratio_mode("vanilla", "lengthnormalisation")
    want = g.solve_with_cost_time_ratio("lawlergpu", 2)
    got = r.solve_with_cost_time_ratio("lawlergpu", 2)
    assert got[0] == want[0] and got[1] == want[1] and np.array_equal(got[2], want[2])
