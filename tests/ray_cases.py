"""Ray casts (World::raycast, riftphys-world/src/world/queries.rs:50-116, through rphys_world_raycast)
over any library exporting the C ABI: the reference's FFI ray tests (riftphys-ffi/src/tests.rs:178-280,
488-530, 1201-1240, 1317-1345) restated, and the batched entry point agreeing with single calls."""
import math

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


# ---- exact rays (World::raycast_exact, queries.rs:18-48, through rphys_ext_raycast_exact_batch)
def _exact(w, o, d, max_d, ignore=None):
    row = w.raycast_batch(np.float32([o]), np.float32([d]), max_d, ignore=ignore, exact=True)[0]
    hit = bool(row[0:1].view(np.uint32)[0])
    return hit, int(row[1:2].view(np.uint32)[0]), float(row[2]), tuple(map(float, row[3:6])), tuple(map(float, row[6:9]))


def _qz(deg):
    h = math.radians(deg) / 2.0
    return (0.0, 0.0, math.sin(h), math.cos(h))


def case_exact_tilted_plate_reads_its_slope_not_its_bounds(lib):
    """raycast_exact_test.rs:15-30: a 10 mm plate tilted 30 degrees; the exact ray reads the top face
    at y = x tan30 + 0.005 / cos30, the AABB ray the top of the bounds."""
    w = lib.world(8, 8)
    w.add_box((0.0, 0.0, 0.0), (0.1, 0.005, 0.1), dynamic=False, q=_qz(30.0))
    for x in (-0.05, 0.0, 0.05):
        hit, _, _, point, _ = _exact(w, (x, 0.5, 0.0), (0.0, -1.0, 0.0), 1.0)
        want = x * math.tan(math.radians(30.0)) + 0.005 / math.cos(math.radians(30.0))
        assert hit and abs(point[1] - want) < 1e-5, (x, point, want)
        ahit, _, _, apoint, _ = w.raycast((x, 0.5, 0.0), (0.0, -1.0, 0.0), 1.0)
        assert ahit and apoint[1] > want - 1e-6
    w.close()


def case_exact_ray_passes_through_a_gap_between_plates(lib):
    """raycast_exact_test.rs:32-48: two plates with a 2 mm gap over a table; the ray through the gap
    hits the table, one beside it the plate, and skipping the table sees through it."""
    w = lib.world(8, 8)
    w.add_box((-0.051, -0.005, 0.0), (0.05, 0.005, 0.1), dynamic=False)
    w.add_box((0.051, -0.005, 0.0), (0.05, 0.005, 0.1), dynamic=False)
    table = w.add_box((0.0, -0.02, 0.0), (0.2, 0.01, 0.2), dynamic=False)
    hit, body, _, point, _ = _exact(w, (0.0, 0.2, 0.0), (0.0, -1.0, 0.0), 1.0)
    assert hit and body == table and abs(point[1] + 0.01) < 1e-6, (body, point)
    hit, _, _, point, _ = _exact(w, (0.0015, 0.2, 0.0), (0.0, -1.0, 0.0), 1.0)
    assert hit and abs(point[1]) < 1e-6
    hit, _, _, _, _ = _exact(w, (0.0, -0.015, 0.0), (0.0, -1.0, 0.0), 1.0, ignore=table)
    assert not hit
    w.close()


def case_exact_capsule_and_sphere_hit_their_surface(lib):
    """raycast_exact_test.rs:50-60 and raycast.rs:153-172: the sphere's surface, not its bounds; a
    capsule's side, its cap from above, and a miss past the cap."""
    w = lib.world(8, 8)
    w.add_sphere((0.0, 0.0, 0.0), 0.1, dynamic=False)
    hit, _, _, point, _ = _exact(w, (0.08, 1.0, 0.0), (0.0, -1.0, 0.0), 2.0)
    assert hit and abs(point[1] - 0.06) < 1e-5, point
    assert not _exact(w, (0.09, 1.0, 0.09), (0.0, -1.0, 0.0), 2.0)[0]
    assert w.raycast((0.09, 1.0, 0.09), (0.0, -1.0, 0.0), 2.0)[0]
    w.close()
    w = lib.world(8, 8)
    w.add_capsule((0.0, 0.0, 0.0), 0.2, 0.5, dynamic=False)
    hit, _, frac, _, _ = _exact(w, (-1.0, 0.3, 0.0), (1.0, 0.0, 0.0), 10.0)
    assert hit and abs(frac * 10.0 - 0.8) < 1e-5
    hit, _, frac, _, normal = _exact(w, (0.0, 2.0, 0.0), (0.0, -1.0, 0.0), 10.0)
    assert hit and abs(frac * 10.0 - 1.3) < 1e-5 and abs(normal[1] - 1.0) < 1e-5
    assert not _exact(w, (-1.0, 0.71, 0.0), (1.0, 0.0, 0.0), 10.0)[0]
    w.close()


def case_exact_starting_inside_hits_at_zero(lib):
    """raycast.rs:174-179: a ray from inside a box hits at t = 0 with normal -dir."""
    w = lib.world(8, 8)
    w.add_box((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), dynamic=False)
    hit, _, frac, point, normal = _exact(w, (0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 5.0)
    assert hit and frac == 0.0 and point == (0.0, 0.0, 0.0) and normal == (-1.0, -0.0, -0.0), (frac, normal)
    w.close()


def case_exact_hits_terrain_with_normal_facing_the_ray(lib):
    """queries.rs:33-41: terrain triangles through ray_shape; the normal faces the ray."""
    w = lib.world(8, 8)
    w.set_heightfield(np.zeros(4, dtype=np.float32), 2, 2, 10.0, 10.0, 0.0, 0.0)
    hit, body, _, point, normal = _exact(w, (1.0, 5.0, 1.0), (0.0, -1.0, 0.0), 50.0)
    assert hit and body == 0xFFFFFFFF and abs(point[1]) < 1e-6 and normal[1] > 0.99, (body, point, normal)
    hit, body, _, _, normal = _exact(w, (1.0, -5.0, 1.0), (0.0, 1.0, 0.0), 50.0)
    assert hit and body == 0xFFFFFFFF and normal[1] < -0.99, normal
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
