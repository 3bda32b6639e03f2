"""The sm_100a solvers against exact known answers (tests/golden/toy_cases.json)."""
import pytest

from test_oracle_golden import CASES, check_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_gpu_matches_known_answers(cpg, c):
    check_case(lambda *a: cpg.product_graph_generator(*a, False, False), c)
