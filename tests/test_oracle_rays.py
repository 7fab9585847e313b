"""Ray casts on the CPU oracle (tests/ray_cases.py). (The same cases, and bit equality with the
oracle, run on the CUDA library in tests/test_gpu_rays.py.)"""
import pytest

import ray_cases as RC


@pytest.mark.parametrize("name", [n for n in dir(RC) if n.startswith("case_")])
def test_case(oracle, name):
    getattr(RC, name)(oracle)
