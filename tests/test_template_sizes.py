"""The layer template built on the host (no GPU): its sizes against the
oracle's product space (the reference's productspace rows), for plain and
conjugate graphs, pruned or not.  An interlayer row joins layer Y edge b to
the next one, so its two leading Y columns differ; an intralayer row stays
on one Y vertex."""
import numpy as np
import pytest

from cyclic_product_graphs import synthetic


@pytest.mark.parametrize("conj", [False, True])
@pytest.mark.parametrize("prune", [False, True])
@pytest.mark.parametrize("level,ny", [(1, 5), (2, 7), (2, 2)])
def test_sizes_match_the_oracle_product_space(cpg, oracle, conj, prune, level, ny):
    p = synthetic.make_pair(icosphere_level=level, n_curve=ny, feat_dim=4, seed=level + ny)
    got = cpg.product_graph_sizes(p["EX"], len(p["VX"]), len(p["EY"]), conj, prune)
    o = oracle.OracleGenerator(p["VX"], p["EX"], p["VY"], p["EY"], p["feat_diff"], conj, False, prune)
    if conj:
        # the product space does not read the normals; a two-point curve has
        # none (its vertex normals cancel), so any unit rows do here
        nx = p.get("NX", np.tile([0.0, 0.0, 1.0], (len(p["VX"]), 1)))
        ny_ = p.get("NY", np.tile([1.0, 0.0, 0.0], (len(p["VY"]), 1)))
        o.set_normals(nx, ny_)
    ps = o.get_product_space()
    assert got["edges"] == ps.shape[0]
    assert got["nodes_per_layer"] == (3 * len(p["EX"]) if conj else len(p["VX"]))
    inter = int(np.count_nonzero(ps[:, 0] != ps[:, 1]))
    assert got["inter_edges_per_block"] * len(p["EY"]) == inter
    assert got["intra_edges_per_block"] * len(p["EY"]) == ps.shape[0] - inter
    assert got["slices"] == (got["nodes_per_layer"] + 31) // 32
    assert got["ell_rows"] * 32 >= got["edges_per_block"]  # padded, holds every edge
    if prune:
        assert got["intra_edges_per_block"] == 0


def test_sizes_reject_out_of_range_edges(cpg):
    with pytest.raises(cpg.PGCError, match="outside VX"):
        cpg.product_graph_sizes(np.array([[0, 5]]), 3, 4)
