"""The host template builder under concurrency, without a GPU: one template
built many times from several threads at once (the worker pool serves one
job, the other callers run inline) equals a single build, byte for byte."""
import os
import subprocess

import numpy as np
import pytest

from cyclic_product_graphs import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def stress(tmp_path_factory):
    out = tmp_path_factory.mktemp("tmpl") / "stress"
    csrc = os.path.join(ROOT, "product-graph-cycles_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc, "-o", str(out),
                    os.path.join(ROOT, "tests", "template_harness", "stress.cpp"),
                    os.path.join(csrc, "graph_template.cpp")], check=True)
    return str(out)


@pytest.mark.parametrize("conj,prune", [(False, False), (True, False), (True, True)])
def test_concurrent_builds_equal_a_single_build(stress, tmp_path, conj, prune):
    p = synthetic.make_pair(n_vertices=2000, n_curve=6, feat_dim=4, seed=1)
    ex = tmp_path / "ex.bin"
    p["EX"].astype(np.int32).tofile(ex)
    r = subprocess.run([stress, str(ex), str(len(p["VX"])), str(int(conj)), str(int(prune)), "7", "6", "8"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("0 of 48 builds differ")
