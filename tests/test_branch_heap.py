"""The branch-and-bound heap of the host driver (csrc/branch_heap.hpp)
against the oracle's restatement of the reference heap
(helper/minheap.cpp:16-277), without a GPU: random operation sequences with
many equal values, pushes of present and out-of-range keys, decreases and
pops, compared result by result.  The pop order of equal lower bounds picks
the next branch, so the two must agree exactly."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def heap(tmp_path_factory):
    out = tmp_path_factory.mktemp("heap") / "heap"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off",
                    "-I", os.path.join(ROOT, "product-graph-cycles_b200", "csrc"), "-I", os.path.join(ROOT, "oracle"),
                    "-o", str(out), os.path.join(ROOT, "tests", "template_harness", "heap.cpp")], check=True)
    return str(out)


@pytest.mark.parametrize("seed,capacity", [(1, 1), (2, 2), (3, 8), (4, 64), (5, 1000)])
def test_heap_matches_the_reference_heap(heap, seed, capacity):
    r = subprocess.run([heap, str(seed), "200000", str(capacity)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("0 of 200000 operations differ")
