"""The reference's W6 bounce acceptance tests (restitution_toi_test.rs) on the CPU oracle. (The same
cases run on the CUDA library in tests/test_gpu_bounce.py.)"""
import pytest

import bounce_cases as B


@pytest.mark.parametrize("name", [n for n in dir(B) if n.startswith("case_")])
def test_case(oracle, name):
    getattr(B, name)(oracle)
