"""W6 bounce passes on the GPU: the reference's restitution acceptance cases (restitution_toi_test.rs,
restated in tests/bounce_cases.py), and tick-by-tick bit parity with the CPU oracle on scenes where
many bodies bounce at once (balls and boxes of rubber and aluminium dropped on each other and on a
rubber floor; a rubber pile with a jointed chain in it)."""
import numpy as np
import pytest

import bounce_cases as BC
from conftest import rp
from test_gpu_parity import run_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", [n for n in dir(BC) if n.startswith("case_")])
def test_case(gpu, name):
    getattr(BC, name)(gpu)


def _bouncers(n, seed, joints=False):
    def build(rp_, w):
        w.set_gravity((0.0, -9.81, 0.0))
        BC._floor(w, BC.RUBBER)
        rng = np.random.default_rng(seed)
        for k in range(n):
            pos = (rng.uniform(-1.5, 1.5), rng.uniform(0.5, 4.0), rng.uniform(-1.5, 1.5))
            vel = (rng.normal() * 0.5, rng.uniform(-3.0, 0.0), rng.normal() * 0.5)
            mat = BC.RUBBER if k % 2 == 0 else BC.ALUMINUM
            if k % 3 == 0:
                BC._ball(w, pos, vel, rng.uniform(0.1, 0.3), rng.uniform(0.2, 3.0), mat)
            else:
                q = rng.normal(size=4)
                q /= np.linalg.norm(q)
                BC._box(w, pos, tuple(rng.uniform(0.08, 0.3, 3)), rng.uniform(0.2, 3.0), mat, rot=tuple(q))
        if joints:  # a hinged pair falling into the pile: its contacts bounce by the restitution pass
            d = rp_.desc_array(np.array([[0.0, 5.0, 0.0], [0.8, 5.0, 0.0]]), np.tile([0.0, 0.0, 0.0, 1.0], (2, 1)),
                               np.full((2, 3), 0.2), rp_.SHAPE_BOX, np.full(2, 800.0), np.ones(2, dtype=np.uint32),
                               material=BC.RUBBER, sleep_allowed=0)
            a = w.add_bodies_array(d)
            w.add_joints([(rp_.JOINT_HINGE, a, a + 1, ((0.4, 0.0, 0.0), (0, 0, 0, 1)), ((-0.4, 0.0, 0.0), (0, 0, 0, 1)), 2)])
        return 1.0 / 60.0, w.num_bodies()
    return build


def test_bouncing_pile(oracle, gpu):
    wo, _ = run_pair(oracle, gpu, {"cap": (64, 64), "fn": _bouncers(30, 1)}, 300)
    assert wo.stats()["bounce_rows"] >= 0


def test_bouncing_pile_with_joints(oracle, gpu):
    run_pair(oracle, gpu, {"cap": (64, 64), "fn": _bouncers(24, 2, joints=True)}, 300)


def test_bouncing_pile_240hz(oracle, gpu):
    def build(rp_, w):
        _bouncers(30, 3)(rp_, w)
        return 1.0 / 240.0, w.num_bodies()
    run_pair(oracle, gpu, {"cap": (64, 64), "fn": build}, 600, check_every=3)
