"""The riftnet wire snapshot on the CPU oracle (tests/wire_cases.py). (The same cases, and byte
equality with the oracle, run on the CUDA library in tests/test_gpu_wire.py.)"""
import pytest

import wire_cases as WC


@pytest.mark.parametrize("name", [n for n in dir(WC) if n.startswith("case_")])
def test_case(oracle, name):
    getattr(WC, name)(oracle)
