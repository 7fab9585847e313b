"""Ray casts (World::raycast, riftphys-world/src/world/queries.rs:50-116, through rphys_world_raycast)
over any library exporting the C ABI: the reference's FFI ray tests (riftphys-ffi/src/tests.rs:178-280,
488-530, 1201-1240, 1317-1345) restated, and the batched entry point agreeing with single calls."""
import numpy as np

from conftest import rp, scenes


def _ground(w):
    return w.add_box((0.0, -0.5, 0.0), (50.0, 0.5, 50.0), dynamic=False)


def case_raycast_hits_ground_box_and_ignore_works(lib):
    """tests.rs:178-224"""
    w = lib.world(8, 8)
    g = _ground(w)
    hit, body, frac, point, normal = w.raycast((0.0, 5.0, 0.0), (0.0, -1.0, 0.0), 20.0)
    assert hit and body == g
    hit2, body2, frac2, _, _ = w.raycast((0.0, 5.0, 0.0), (0.0, -1.0, 0.0), 20.0, ignore=g)
    assert not hit2 and body2 == 0 and frac2 == 1.0
    w.close()


def case_raycast_zero_direction_is_safe_and_misses(lib):
    """tests.rs:226-252"""
    w = lib.world(8, 8)
    _ground(w)
    hit, body, frac, point, normal = w.raycast((0.0, 5.0, 0.0), (0.0, 0.0, 0.0), 20.0)
    assert not hit and body == 0 and frac == 1.0 and normal == (0.0, 1.0, 0.0)
    w.close()


def case_raycast_invalid_ignore_returns_invalid_id(lib):
    """tests.rs:254-280: an out-of-range ignore_body is RPHYS_ERR_INVALID_ID."""
    w = lib.world(8, 8)
    try:
        w.raycast((0.0, 5.0, 0.0), (0.0, -1.0, 0.0), 20.0, ignore=999999)
    except rp.RPhysError as e:
        assert "0x2" in str(e), str(e)
    else:
        raise AssertionError("an invalid ignore_body was accepted")
    w.close()


def case_raycast_hits_terrain_when_heightfield_enabled(lib):
    """tests.rs:488-530: a flat 2 x 2 heightfield of 10 m cells, a ray straight down hits it at y = 0
    with an upward normal and the terrain's id."""
    w = lib.world(8, 8)
    w.set_heightfield(np.zeros(4, dtype=np.float32), 2, 2, 10.0, 10.0, 0.0, 0.0)
    hit, body, frac, point, normal = w.raycast((1.0, 5.0, 1.0), (0.0, -1.0, 0.0), 50.0)
    assert hit and body == 0xFFFFFFFF and abs(point[1]) < 1e-3 and normal[1] > 0.9, (hit, body, point, normal)
    w.close()


def case_raycast_fraction_is_in_0_1_on_hit_and_1_on_miss(lib):
    """tests.rs:1201-1240"""
    w = lib.world(8, 8)
    _ground(w)
    hit, _, frac, _, _ = w.raycast((0.0, 5.0, 0.0), (0.0, -1.0, 0.0), 20.0)
    assert hit and 0.0 <= frac <= 1.0 and abs(frac - 0.25) < 1e-6
    miss, _, frac2, _, _ = w.raycast((0.0, 5.0, 0.0), (0.0, 1.0, 0.0), 20.0)
    assert not miss and frac2 == 1.0
    w.close()


def case_raycast_negative_max_distance_is_safe_and_misses(lib):
    """tests.rs:1317-1345"""
    w = lib.world(8, 8)
    _ground(w)
    hit, body, frac, _, _ = w.raycast((0.0, 5.0, 0.0), (0.0, -1.0, 0.0), -3.0)
    assert not hit and body == 0 and frac == 1.0
    w.close()


def stepped_terrain(lib):
    w = lib.world(2048, 2048)
    scenes.terrain(rp, w, n_bodies=1500, hf_n=96, area=80.0)
    for _ in range(60):
        w.step(1.0 / 60.0)
    return w


def random_rays(n, seed):
    rng = np.random.default_rng(seed)
    o = np.column_stack([rng.uniform(-45, 45, n), rng.uniform(5, 40, n), rng.uniform(-45, 45, n)]).astype(np.float32)
    d = np.column_stack([rng.normal(size=n), -np.abs(rng.normal(size=n)) - 0.2, rng.normal(size=n)]).astype(np.float32)
    d[::17] = 0.0  # some zero directions: misses
    return o, d


def case_batched_rays_equal_single_calls(lib):
    w = stepped_terrain(lib)
    o, d = random_rays(300, 4)
    out = w.raycast_batch(o, d, 80.0)
    for i in range(0, 300, 7):
        hit, body, frac, point, normal = w.raycast(tuple(o[i]), tuple(d[i]), 80.0)
        row = out[i]
        assert bool(row[0:1].view(np.uint32)[0]) == hit and int(row[1:2].view(np.uint32)[0]) == body
        assert np.array_equal(np.float32([frac, *point, *normal]), row[2:9]), (i, row, frac, point, normal)
    assert out[:, 0].view(np.uint32).sum() > 100  # most rays hit something
    w.close()


# ---- capsule sweeps (World::sweep_capsule, queries.rs:118-249, through rphys_world_capsule_sweep)
def case_capsule_sweep_hits_wall_and_ignore_works(lib):
    """tests.rs:282-330"""
    w = lib.world(8, 8)
    wall = w.add_box((3.0, 1.0, 0.0), (0.125, 2.0, 2.0), dynamic=False)
    hit, body, frac, over, point, normal = w.capsule_sweep((0.0, 1.0, 0.0), (6.0, 1.0, 0.0), 0.5, 0.5)
    assert hit and body == wall and 0.0 <= frac <= 1.0 and not over
    hit2, body2, frac2, _, _, _ = w.capsule_sweep((0.0, 1.0, 0.0), (6.0, 1.0, 0.0), 0.5, 0.5, ignore=wall)
    assert not hit2 and body2 == 0 and frac2 == 1.0
    w.close()


def case_capsule_sweep_invalid_ignore_returns_invalid_id(lib):
    """tests.rs:829-860"""
    w = lib.world(8, 8)
    try:
        w.capsule_sweep((0.0, 1.0, 0.0), (6.0, 1.0, 0.0), 0.5, 0.5, ignore=999999)
    except rp.RPhysError as e:
        assert "0x2" in str(e), str(e)
    else:
        raise AssertionError("an invalid ignore_body was accepted")
    w.close()


def case_capsule_sweep_started_overlapping_sets_flag(lib):
    """tests.rs:1344-1380"""
    w = lib.world(8, 8)
    wall = w.add_box((0.0, 1.0, 0.0), (1.0, 1.0, 1.0), dynamic=False)
    hit, body, frac, over, _, _ = w.capsule_sweep((0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 0.75, 0.5)
    assert hit and body == wall and over and 0.0 <= frac <= 1.0
    w.close()


def case_capsule_sweep_argument_checks(lib):
    w = lib.world(8, 8)
    for args in (((float("nan"), 0, 0), (1, 0, 0), 0.5, 0.5), ((0, 0, 0), (1, 0, 0), 0.0, 0.5),
                 ((0, 0, 0), (1, 0, 0), 0.5, -1.0)):
        try:
            w.capsule_sweep(*args)
        except rp.RPhysError:
            pass
        else:
            raise AssertionError(f"accepted {args}")
    w.close()


def random_sweeps(n, seed):
    rng = np.random.default_rng(seed)
    frm = np.column_stack([rng.uniform(-40, 40, n), rng.uniform(2, 20, n), rng.uniform(-40, 40, n)])
    to = frm + np.column_stack([rng.normal(size=n) * 6, -np.abs(rng.normal(size=n)) * 10, rng.normal(size=n) * 6])
    to[::13] = frm[::13]  # stationary
    r = rng.uniform(0.1, 0.6, n)
    hh = rng.uniform(0.0, 0.8, n)
    return frm, to, r, hh
