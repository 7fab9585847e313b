"""The player controller on the GPU (one block runs the players in order): the cases of
tests/player_cases.py, and every tick's player poses, grounded flags and world hash bit for bit the
oracle's with players walking into terrain, bodies and one another."""
import struct

import pytest

import player_cases as PC

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", [n for n in dir(PC) if n.startswith("case_")])
def test_case(gpu, name):
    getattr(PC, name)(gpu)


def _bits(poses):
    return [(struct.pack("<7f", *p, *q), g) for p, q, g in poses]


def test_players_equal_the_oracle(oracle, gpu):
    a, b = PC.crowd(oracle), PC.crowd(gpu)
    grounded = 0
    for t, ((pa, ha), (pb, hb)) in enumerate(zip(a, b)):
        assert _bits(pa) == _bits(pb), (t, pa, pb)
        assert ha == hb, t
        grounded += sum(g for _, _, g in pa)
    assert grounded > 0
