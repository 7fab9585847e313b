"""The riftnet wire snapshot packed on the GPU: the cases of tests/wire_cases.py, and the bytes equal
to the oracle's after both step the same terrain scene."""
import pytest

import wire_cases as WC
from conftest import rp, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", [n for n in dir(WC) if n.startswith("case_")])
def test_case(gpu, name):
    getattr(WC, name)(gpu)


def test_snapshot_bytes_equal_the_oracle(oracle, gpu):
    wo, wg = oracle.world(2048, 2048), gpu.world(2048, 2048)
    for w in (wo, wg):
        scenes.terrain(rp, w, n_bodies=1500, hf_n=96, area=80.0)
    for t in range(60):
        wo.step(1.0 / 60.0)
        wg.step(1.0 / 60.0)
    wg.remove_body(7)
    wo.remove_body(7)
    do, co = wo.pack_snapshot(60, 9)
    dg, cg = wg.pack_snapshot(60, 9)
    assert co == cg and do == dg
