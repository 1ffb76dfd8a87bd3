"""Pin the CPU restatement against viprs's golden fixtures and known-answer tests."""
import numpy as np
import pytest

from golden_cases import CASES, expected
from oracle_chain import run_chain


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden_fixture(oracle, name):
    build, chain, shape, tol = CASES[name]
    out = run_chain(build(), chain)
    exp = expected(name, shape)
    assert out.shape == exp.shape
    diff = np.abs(out.astype(np.int32) - exp.astype(np.int32)).max()
    assert diff <= tol, f"{name}: max diff {diff} > {tol}"
