"""The kinematic player controller (World::update_players, riftphys-world/src/world/step.rs:544-639,
through rphys_add_player / rphys_player_set_input / rphys_player_get_pose, lib.rs:1580-1693) over any
library exporting the C ABI: the reference's FFI player tests (riftphys-ffi/src/tests.rs:1514-1611)
restated, the argument checks of lib.rs, and a players-in-a-crowd scene both libraries step alike."""
import numpy as np

from conftest import rp, scenes


def _expect(code, fn, *args):
    try:
        fn(*args)
    except rp.RPhysError as e:
        assert e.code == code, str(e)
    else:
        raise AssertionError(f"expected error {code:#x}")


def case_player_basic_movement_and_gravity(lib):
    """tests.rs:1514-1559: in the air with input +X, ten ticks fall and move it, not grounded."""
    w = lib.world(64, 64)
    p = w.add_player(rp.iso(0.0, 10.0, 0.0), 0.4, 1.8, 5.0)
    assert p == 0
    w.player_set_input(p, (1.0, 0.0, 0.0))
    for _ in range(10):
        w.step(1.0 / 60.0)
    pos, rot, grounded = w.player_pose(p)
    assert pos[1] < 10.0 and pos[0] > 0.0 and not grounded, (pos, grounded)
    assert rot == (0.0, 0.0, 0.0, 1.0)
    w.close()


def case_player_hits_heightfield_and_grounds(lib):
    """tests.rs:1561-1611: a flat 2 x 2 heightfield of 10 m cells; a player of radius 0.5 and height
    2 dropped from y = 3 settles grounded at y in (1.4, 1.6)."""
    w = lib.world(64, 64)
    w.set_heightfield(np.zeros(4, dtype=np.float32), 2, 2, 10.0, 10.0, 0.0, 0.0)
    p = w.add_player(rp.iso(5.0, 3.0, 5.0), 0.5, 2.0, 5.0)
    for _ in range(60):
        w.step(1.0 / 60.0)
    pos, _, grounded = w.player_pose(p)
    assert grounded and 1.4 < pos[1] < 1.6, (pos, grounded)
    w.close()


def case_player_argument_checks(lib):
    """lib.rs:1580-1693: bad sizes, non-finite poses and inputs, indices out of range, capacity."""
    w = lib.world(2, 2)
    _expect(rp.RPHYS_ERR_BAD_ARG, w.add_player, rp.iso(0.0, 1.0, 0.0), 0.0, 1.8, 5.0)
    _expect(rp.RPHYS_ERR_BAD_ARG, w.add_player, rp.iso(0.0, 1.0, 0.0), 0.4, -1.0, 5.0)
    _expect(rp.RPHYS_ERR_BAD_ARG, w.add_player, rp.iso(float("nan"), 1.0, 0.0), 0.4, 1.8, 5.0)
    _expect(rp.RPHYS_ERR_BAD_ARG, w.player_set_input, 0, (1.0, 0.0, 0.0))
    _expect(rp.RPHYS_ERR_BAD_ARG, w.player_pose, 0)
    a = w.add_player(rp.iso(0.0, 1.0, 0.0))
    b = w.add_player(rp.iso(3.0, 1.0, 0.0))
    assert (a, b) == (0, 1)
    _expect(rp.RPHYS_ERR_CAPACITY, w.add_player, rp.iso(6.0, 1.0, 0.0))
    _expect(rp.RPHYS_ERR_BAD_ARG, w.player_set_input, 1, (float("inf"), 0.0, 0.0))
    _expect(rp.RPHYS_ERR_BAD_ARG, w.player_set_input, 2, (1.0, 0.0, 0.0))
    _expect(rp.RPHYS_ERR_BAD_ARG, w.player_pose, 2)
    # the player's body is a real body: id a + 1, static, with the start pose
    pos, _ = w.pose(1)
    assert pos == (0.0, 1.0, 0.0)
    w.close()


def case_player_kicks_a_dynamic_body(lib):
    """step.rs:620-627: walking into a resting dynamic sphere wakes it and kicks it (an impulse of
    -n * 10, n the narrowphase normal from the player's capsule to the sphere); it was at rest before."""
    w = lib.world(16, 16)
    w.add_box((0.0, -0.5, 0.0), (20.0, 0.5, 20.0), dynamic=False)
    s = w.add_sphere((2.0, 0.5, 0.0), 0.5, mass=1.0)
    p = w.add_player(rp.iso(0.0, 0.95, 0.0), 0.4, 1.8, 5.0)
    w.player_set_input(p, (1.0, 0.0, 0.0))
    vx = []
    for _ in range(40):
        w.step(1.0 / 60.0)
        vx.append(w.velocity(s)[0][0])
    assert vx[0] == 0.0 and max(abs(v) for v in vx) > 0.1, vx
    pos, _, grounded = w.player_pose(p)
    assert grounded and pos[0] > 0.3 and all(np.isfinite(pos)), (pos, grounded)
    w.close()


def case_player_snapshot_restore_replays(lib):
    """lib.rs:1696-1793: the snapshot carries the controllers; a restore then the same ticks give the
    same poses and grounded flags."""
    w = lib.world(64, 64)
    w.set_heightfield(np.zeros(4, dtype=np.float32), 2, 2, 10.0, 10.0, 0.0, 0.0)
    p = w.add_player(rp.iso(5.0, 3.0, 5.0), 0.5, 2.0, 5.0)
    w.player_set_input(p, (0.3, 0.0, 1.0))
    for _ in range(20):
        w.step(1.0 / 60.0)
    snap = w.snapshot()
    runs = []
    for _ in range(2):
        w.restore(snap)
        seq = []
        for _ in range(25):
            w.step(1.0 / 60.0)
            seq.append(w.player_pose(p))
        runs.append(seq)
    assert runs[0] == runs[1]
    w.free_snapshot(snap)
    w.close()


def crowd(lib, ticks=90, n_players=8, n_bodies=600):
    """Players walking and falling through the stepped terrain scene and into one another: per tick
    every player's pose and grounded flag and the world's hash."""
    w = lib.world(n_bodies + 64, n_bodies + 64)
    scenes.terrain(rp, w, n_bodies=n_bodies, hf_n=64, area=50.0)
    rng = np.random.default_rng(7)
    ps = []
    for i in range(n_players):
        # pairs of players side by side, facing one another, some starting in the air
        x, z = float(rng.uniform(-15, 15)), float(rng.uniform(-15, 15))
        y = 4.0 + 1.5 * (i % 3)
        a = w.add_player(rp.iso(x, y, z), 0.4 + 0.05 * (i % 2), 1.6 + 0.2 * (i % 3), 4.0 + i)
        b = w.add_player(rp.iso(x + 1.2, y, z), 0.4, 1.8, 5.0)
        w.player_set_input(a, (1.0, 0.0, float(rng.normal())))
        w.player_set_input(b, (-1.0, 0.0, 0.0))
        ps += [a, b]
    out = []
    for t in range(ticks):
        if t == ticks // 2:
            for i in ps[::3]:
                w.player_set_input(i, (float(rng.normal()), 0.0, float(rng.normal())))
        w.step(1.0 / 60.0)
        poses = [w.player_pose(i) for i in ps]
        out.append((poses, w.hash()))
    w.close()
    return out


def case_players_in_a_crowd_stay_sane(lib):
    out = crowd(lib, ticks=30, n_players=3, n_bodies=200)
    poses = out[-1][0]
    for pos, rot, _ in poses:
        assert all(np.isfinite(pos)) and rot == (0.0, 0.0, 0.0, 1.0)
    assert any(g for _, _, g in poses)
