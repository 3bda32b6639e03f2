"""The product space that the host layer template defines (the rows the
library returns, and every edge's source and target node) against the fixture
script's restatements of product_space.cpp and conj_product_space.cpp, and
its sliced-ELL in-edge lists against its own edge list, without a GPU:
plain, pruned, conjugate and pruned conjugate graphs, 2 to 5 layers, on the
toy meshes and on a 400-vertex synthetic mesh."""
import os
import subprocess
import sys

import numpy as np
import pytest

from cyclic_product_graphs import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden  # noqa: E402


@pytest.fixture(scope="module")
def rows_tool(tmp_path_factory):
    out = tmp_path_factory.mktemp("rows") / "rows"
    csrc = os.path.join(ROOT, "product-graph-cycles_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc, "-o", str(out),
                    os.path.join(ROOT, "tests", "template_harness", "rows.cpp"),
                    os.path.join(csrc, "graph_template.cpp")], check=True)
    return str(out)


def _meshes():
    out = [(name, make_golden.directed(und), len(V)) for name, (V, und) in make_golden.MESHES.items()]
    p = synthetic.make_pair(n_vertices=400, n_curve=6, feat_dim=4, seed=5)
    out.append(("synthetic400", p["EX"].astype(np.int32), len(p["VX"])))
    return out


@pytest.fixture(scope="module")
def ell_tool(tmp_path_factory):
    out = tmp_path_factory.mktemp("ell") / "ell"
    csrc = os.path.join(ROOT, "product-graph-cycles_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc, "-o", str(out),
                    os.path.join(ROOT, "tests", "template_harness", "ell.cpp"),
                    os.path.join(csrc, "graph_template.cpp")], check=True)
    return str(out)


@pytest.mark.parametrize("ny", [2, 3, 5])
@pytest.mark.parametrize("kind", ["plain", "plain_pruned", "conj", "conj_pruned"])
@pytest.mark.parametrize("mesh", _meshes(), ids=lambda m: m[0])
def test_in_edge_lists_hold_every_edge_once_in_tie_order(ell_tool, tmp_path, mesh, kind, ny):
    _, EX, nvx = mesh
    EY = np.stack([np.arange(ny), (np.arange(ny) + 1) % ny], axis=1).astype(np.int32)
    EX.astype(np.int32).tofile(tmp_path / "ex.bin")
    EY.tofile(tmp_path / "ey.bin")
    r = subprocess.run([ell_tool, str(tmp_path / "ex.bin"), str(tmp_path / "ey.bin"), str(nvx),
                        str(int(kind.startswith("conj"))), str(int(kind.endswith("pruned")))],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("0 problems")


@pytest.mark.parametrize("ny", [2, 3, 5])
@pytest.mark.parametrize("kind", ["plain", "plain_pruned", "conj", "conj_pruned"])
@pytest.mark.parametrize("mesh", _meshes(), ids=lambda m: m[0])
def test_template_product_space_matches_the_restatement(rows_tool, tmp_path, mesh, kind, ny):
    _, EX, nvx = mesh
    EY = np.stack([np.arange(ny), (np.arange(ny) + 1) % ny], axis=1).astype(np.int32)
    conj, prune = kind.startswith("conj"), kind.endswith("pruned")
    if conj:
        ps, src, trgt = make_golden.conj_product(EX, EY, prune)
    else:
        ps, src, trgt = make_golden.plain_product(EX, EY, nvx, prune)
    EX.astype(np.int32).tofile(tmp_path / "ex.bin")
    EY.tofile(tmp_path / "ey.bin")
    out = tmp_path / "out.bin"
    r = subprocess.run([rows_tool, str(tmp_path / "ex.bin"), str(tmp_path / "ey.bin"), str(nvx), str(int(conj)),
                        str(int(prune)), str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(out, dtype="<i4")
    e, c = ps.shape
    assert got.size == e * c + 2 * e
    assert np.array_equal(got[:e * c].reshape(e, c), ps)
    assert np.array_equal(got[e * c:e * c + e], np.asarray(src))
    assert np.array_equal(got[e * c + e:], np.asarray(trgt))
