"""The Bellman-Ford team's CTA slice ranges, without a GPU: for every
(K, warps, blocks) of a grid, the planner's contiguous ranges reach the
smallest step cost that any partition of the template's slices into at most
`blocks` ranges has under the same cost model (exact search by dynamic
programming over every intralayer bound), and the team's wait lists equal
the CTA pairs that the template's edges join."""
import os
import subprocess

import numpy as np
import pytest

from cyclic_product_graphs import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def cuts(tmp_path_factory):
    out = tmp_path_factory.mktemp("cuts") / "cuts"
    csrc = os.path.join(ROOT, "product-graph-cycles_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc, "-o", str(out),
                    os.path.join(ROOT, "tests", "template_harness", "cuts.cpp"),
                    os.path.join(csrc, "graph_template.cpp")], check=True)
    return str(out)


@pytest.mark.parametrize("n_vertices,conj,prune", [(1000, False, False), (80, True, False), (300, True, False),
                                                   (600, True, True)])
def test_cuts_reach_the_best_partition(cuts, tmp_path, n_vertices, conj, prune):
    p = synthetic.make_pair(n_vertices=n_vertices, n_curve=6, feat_dim=4, seed=3)
    ex = tmp_path / "ex.bin"
    p["EX"].astype(np.int32).tofile(ex)
    r = subprocess.run([cuts, str(ex), str(len(p["VX"])), str(int(conj)), str(int(prune)), "5"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("0 of 144 plans differ from the best, 0 wait lists differ")
