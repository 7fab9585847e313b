"""Ray casts on the GPU (one block per ray): the cases of tests/ray_cases.py, and every result bit for
bit the oracle's on a stepped terrain scene (colliders' AABBs and heightfield triangles, rays that
miss, start inside, or graze)."""
import numpy as np
import pytest

import ray_cases as RC

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", [n for n in dir(RC) if n.startswith("case_")])
def test_case(gpu, name):
    getattr(RC, name)(gpu)


def test_rays_equal_the_oracle(oracle, gpu):
    wo, wg = RC.stepped_terrain(oracle), RC.stepped_terrain(gpu)
    o, d = RC.random_rays(2000, 11)
    ro = wo.raycast_batch(o, d, 90.0, ignore=5)
    rg = wg.raycast_batch(o, d, 90.0, ignore=5)
    assert np.array_equal(ro.view(np.uint32), rg.view(np.uint32))
    assert ro[:, 0].view(np.uint32).sum() > 1000
