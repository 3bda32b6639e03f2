"""The sm_100a solvers against the known answers on irregular, pruned and
conjugate graphs (tests/golden/mesh_cases.json, pruned_cases.json,
conj_cases.json): product space digests, objectives against their own cycles
and bounded below by the exact optima, exact minimum costs where the
reference's search reaches them, and the reference's NaN ratio where its
initial bound starts from a node without a usable out-edge.  The file sorts
after the other GPU test files (and before the no-allocation test), so a
run that stops at its first failure has run those already."""
import pytest

from test_oracle_golden import BOUNDED_PLAIN_CASES, CONJ_CASES, check_bounded_plain_case, check_conj_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("c", BOUNDED_PLAIN_CASES, ids=[c["name"] for c in BOUNDED_PLAIN_CASES])
def test_gpu_matches_bounded_plain_known_answers(cpg, c):
    check_bounded_plain_case(cpg.product_graph_generator, c)


@pytest.mark.parametrize("c", CONJ_CASES, ids=[c["name"] for c in CONJ_CASES])
def test_gpu_matches_conjugate_known_answers(cpg, c):
    check_conj_case(cpg.product_graph_generator, c)
