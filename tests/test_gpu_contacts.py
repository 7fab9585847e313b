"""rphys_world_get_contacts on the GPU: the cases of tests/contact_cases.py, and the events equal to the
CPU restatement's, byte for byte, on the terrain scene."""
import pytest

import contact_cases as CC
from conftest import rp, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", [n for n in dir(CC) if n.startswith("case_")])
def test_case(gpu, name):
    getattr(CC, name)(gpu)


def test_events_equal_the_oracle(oracle, gpu):
    wo, wg = oracle.world(2048, 2048), gpu.world(2048, 2048)
    for w in (wo, wg):
        scenes.terrain(rp, w, n_bodies=1500, hf_n=96, area=80.0)
    for t in range(90):
        wo.step(1.0 / 60.0)
        wg.step(1.0 / 60.0)
        if t % 15 == 14:
            eo, eg = wo.contacts(), wg.contacts()
            assert len(eo) == len(eg) > 0
            assert b"".join(bytes(e) for e in eo) == b"".join(bytes(e) for e in eg), f"tick {t}: events differ"
