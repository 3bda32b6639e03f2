"""The sm_100a solvers against exact known answers (tests/golden/toy_cases.json,
tests/golden/mesh_cases.json, tests/golden/pruned_cases.json,
tests/golden/conj_cases.json)."""
import pytest

from test_oracle_golden import BOUNDED_PLAIN_CASES, CASES, CONJ_CASES, check_bounded_plain_case, check_case, check_conj_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_gpu_matches_known_answers(cpg, c):
    check_case(lambda *a: cpg.product_graph_generator(*a, False, False), c)


@pytest.mark.parametrize("c", CONJ_CASES, ids=[c["name"] for c in CONJ_CASES])
def test_gpu_matches_conjugate_known_answers(cpg, c):
    check_conj_case(cpg.product_graph_generator, c)


@pytest.mark.parametrize("c", BOUNDED_PLAIN_CASES, ids=[c["name"] for c in BOUNDED_PLAIN_CASES])
def test_gpu_matches_bounded_plain_known_answers(cpg, c):
    check_bounded_plain_case(cpg.product_graph_generator, c)
