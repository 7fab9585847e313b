"""The player controller on the CPU oracle (tests/player_cases.py). (The same cases, and bit equality
with the oracle, run on the CUDA library in tests/test_gpu_players.py.)"""
import pytest

import player_cases as PC


@pytest.mark.parametrize("name", [n for n in dir(PC) if n.startswith("case_")])
def test_case(oracle, name):
    getattr(PC, name)(oracle)
