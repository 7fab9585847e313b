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


def test_capsule_sweeps_equal_the_oracle(oracle, gpu):
    wo, wg = RC.stepped_terrain(oracle), RC.stepped_terrain(gpu)
    frm, to, r, hh = RC.random_sweeps(400, 12)
    hits = 0
    for i in range(400):
        a = wo.capsule_sweep(tuple(frm[i]), tuple(to[i]), float(r[i]), float(hh[i]), ignore=3)
        b = wg.capsule_sweep(tuple(frm[i]), tuple(to[i]), float(r[i]), float(hh[i]), ignore=3)
        fa = np.float32([a[2], *a[4], *a[5]]).view(np.uint32)
        fb = np.float32([b[2], *b[4], *b[5]]).view(np.uint32)
        assert a[:2] == b[:2] and a[3] == b[3] and np.array_equal(fa, fb), (i, a, b)
        hits += a[0]
    assert hits > 100


def test_exact_rays_equal_the_oracle(oracle, gpu):
    wo, wg = RC.stepped_terrain(oracle), RC.stepped_terrain(gpu)
    o, d = RC.random_rays(2000, 13)
    ro = wo.raycast_batch(o, d, 90.0, ignore=5, exact=True)
    rg = wg.raycast_batch(o, d, 90.0, ignore=5, exact=True)
    assert np.array_equal(ro.view(np.uint32), rg.view(np.uint32))
    hits = ro[:, 0].view(np.uint32)
    assert hits.sum() > 1000
    # some rays end on bodies, not only on the terrain
    assert (ro[:, 1].view(np.uint32)[hits == 1] != 0xFFFFFFFF).sum() > 50
