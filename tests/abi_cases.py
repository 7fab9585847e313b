"""Contract, determinism and acceptance cases of the reference's test suite, written once against
the C ABI and run on any library exporting it: the CPU oracle (tests/test_oracle_*.py) and the CUDA
product (tests/test_gpu_abi.py). Each case cites the reference test it ports."""
import ctypes
import math
import threading
from ctypes import byref, c_char_p, c_float, c_uint32, c_uint64

import numpy as np

from conftest import rp, scenes

DT = 1.0 / 60.0


def mk_world(lib):
    # crates/riftphys-ffi/src/tests.rs:17-27
    w = lib.world(1024, 2048)
    w.c("rphys_world_set_epoch", c_uint64(1))
    w.c("rphys_world_set_rng_seed", c_uint64(0xBADC0FFE))
    return w


def box_desc(pos, he, dynamic=True, mass=1.0, q=(0, 0, 0, 1)):
    return rp.BoxBodyDesc(rp.iso(*pos, q=q), rp.vel(), he[0], he[1], he[2], mass,
                          rp.RPHYS_BODY_DYNAMIC if dynamic else rp.RPHYS_BODY_STATIC, rp.Material(0.9, 0.7, 0.0), 0)


def sphere_desc(pos, r, dynamic=True, mass=1.0):
    return rp.SphereBodyDesc(rp.iso(*pos), rp.vel(), r, mass,
                             rp.RPHYS_BODY_DYNAMIC if dynamic else rp.RPHYS_BODY_STATIC, rp.Material(0.9, 0.7, 0.0), 0)


def raw(lib, name, *args):
    return getattr(lib.dll, name)(*args)


# ------------------------------------------------------------------ ABI basics (tests.rs:61-142, 1416-1432)
def case_abi_version_and_build_id(lib):
    assert lib.dll.rphys_get_abi_version() == 1
    assert b"riftphys_ffi-" in lib.dll.rphys_get_build_id()


def case_abi_layout_sizes(lib):
    assert ctypes.sizeof(rp.Vec3) == 12 and ctypes.sizeof(rp.Quat) == 16
    assert ctypes.sizeof(rp.Isometry) == 28 and ctypes.sizeof(rp.Velocity) == 24
    assert ctypes.sizeof(rp.Hash32) == 32 and ctypes.sizeof(rp.StepParams) == 20
    assert ctypes.sizeof(rp.ContactEvent) == 36


def case_step_ex_rejects_bad_params(lib):
    w = mk_world(lib)
    p = rp.StepParams(ctypes.sizeof(rp.StepParams) - 1, 0, 1, 0, DT)
    assert raw(lib, "rphys_world_step_ex", w.h, byref(p)) == rp.RPHYS_ERR_BAD_ARG
    p = rp.StepParams(ctypes.sizeof(rp.StepParams), 0, 0, 0, DT)
    assert raw(lib, "rphys_world_step_ex", w.h, byref(p)) == rp.RPHYS_ERR_BAD_ARG
    for dt in (float("nan"), float("inf"), -DT):
        p = rp.StepParams(ctypes.sizeof(rp.StepParams), 0, 1, 0, dt)
        assert raw(lib, "rphys_world_step_ex", w.h, byref(p)) == rp.RPHYS_ERR_BAD_ARG
    assert raw(lib, "rphys_world_step_ex", None, byref(p)) == rp.RPHYS_ERR_NULL


def case_tick_index_with_substeps(lib):
    # tests.rs:863-889
    w = mk_world(lib)
    assert w.tick() == 0
    w.step(DT)
    assert w.tick() == 1
    w.step(DT, substeps=4)
    assert w.tick() == 5


def case_sphere_integrates_downward(lib):
    # tests.rs:144-176
    w = mk_world(lib)
    sid = w.add_sphere((0, 10, 0), 0.5)
    w.step(DT)
    v, _ = w.velocity(sid)
    assert v[1] < 0.0
    p, _ = w.pose(sid)
    assert p[1] < 10.0


def case_terrain_sentinel_rejected(lib):
    # tests.rs:535-590
    w = mk_world(lib)
    w.add_sphere((0, 1, 0), 0.5)
    T = rp.RPHYS_TERRAIN_BODY_ID
    pose = rp.Isometry()
    vel = rp.Velocity()
    assert raw(lib, "rphys_body_get_pose", w.h, T, byref(pose)) == rp.RPHYS_ERR_INVALID_ID
    assert (pose.rot.w, pose.pos.x) == (1.0, 0.0)  # deterministic default written first
    assert raw(lib, "rphys_body_set_pose", w.h, T, byref(rp.iso())) == rp.RPHYS_ERR_INVALID_ID
    assert raw(lib, "rphys_body_get_velocity", w.h, T, byref(vel)) == rp.RPHYS_ERR_INVALID_ID
    assert raw(lib, "rphys_body_set_velocity", w.h, T, byref(rp.vel())) == rp.RPHYS_ERR_INVALID_ID
    assert raw(lib, "rphys_body_apply_impulse", w.h, T, rp.Vec3(0, 1, 0)) == rp.RPHYS_ERR_INVALID_ID
    assert raw(lib, "rphys_body_remove", w.h, T) == rp.RPHYS_ERR_INVALID_ID
    assert raw(lib, "rphys_body_get_pose", w.h, 0, byref(pose)) == rp.RPHYS_ERR_INVALID_ID


def case_ids_monotonic_never_reused(lib):
    # tests.rs:648-759, 1286-1315, 1465-1496
    w = mk_world(lib)
    a = w.add_sphere((0, 1, 0), 0.5)
    b = w.add_sphere((2, 1, 0), 0.5)
    assert (a, b) == (1, 2)
    assert raw(lib, "rphys_body_remove", w.h, a) == rp.RPHYS_OK
    assert raw(lib, "rphys_body_remove", w.h, a) == rp.RPHYS_ERR_INVALID_ID
    c = w.add_sphere((4, 1, 0), 0.5)
    assert c == 3
    pose = rp.Isometry()
    assert raw(lib, "rphys_body_get_pose", w.h, a, byref(pose)) == rp.RPHYS_ERR_INVALID_ID
    for _ in range(20):
        w.add_sphere((0, 5, 0), 0.2)
    assert raw(lib, "rphys_body_get_pose", w.h, a, byref(pose)) == rp.RPHYS_ERR_INVALID_ID
    n = c_uint32(0)
    w.c("rphys_world_num_bodies", byref(n))
    assert n.value == 23


def case_capacity_errors(lib):
    # tests.rs:761-795, 1012-1041
    w = lib.world(2, 8)
    w.add_sphere((0, 1, 0), 0.5)
    w.add_sphere((2, 1, 0), 0.5)
    out = c_uint32(7)
    d = sphere_desc((0, 3, 0), 0.5)
    assert raw(lib, "rphys_add_sphere_body", w.h, byref(d), byref(out)) == rp.RPHYS_ERR_CAPACITY
    assert out.value == 0
    w2 = lib.world(8, 1)
    w2.add_sphere((0, 1, 0), 0.5)
    assert raw(lib, "rphys_add_sphere_body", w2.h, byref(d), byref(out)) == rp.RPHYS_ERR_CAPACITY


def case_null_args_and_bad_shapes(lib):
    # tests.rs:797-827, 1043-1149
    w = mk_world(lib)
    out = c_uint32(9)
    assert raw(lib, "rphys_add_sphere_body", None, byref(sphere_desc((0, 1, 0), 1)), byref(out)) == rp.RPHYS_ERR_NULL
    assert out.value == 0
    assert raw(lib, "rphys_add_sphere_body", w.h, None, byref(out)) == rp.RPHYS_ERR_NULL
    for r in (0.0, -1.0, float("nan"), float("inf")):
        assert raw(lib, "rphys_add_sphere_body", w.h, byref(sphere_desc((0, 1, 0), r)), byref(out)) == rp.RPHYS_ERR_BAD_ARG
    for he in ((0, 1, 1), (1, -1, 1), (1, 1, float("nan"))):
        assert raw(lib, "rphys_add_box_body", w.h, byref(box_desc((0, 1, 0), he)), byref(out)) == rp.RPHYS_ERR_BAD_ARG
    cap = rp.CapsuleBodyDesc(rp.iso(), rp.vel(), 0.2, -0.1, 1.0, 1, rp.Material(0.5, 0.5, 0), 0)
    assert raw(lib, "rphys_add_capsule_body", w.h, byref(cap), byref(out)) == rp.RPHYS_ERR_BAD_ARG
    d = sphere_desc((0, 1, 0), 0.5, mass=0.0)
    assert raw(lib, "rphys_add_sphere_body", w.h, byref(d), byref(out)) == rp.RPHYS_ERR_BAD_ARG
    sid = w.add_sphere((0, 1, 0), 0.5)
    bad = rp.iso(float("nan"), 0, 0)
    assert raw(lib, "rphys_body_set_pose", w.h, sid, byref(bad)) == rp.RPHYS_ERR_BAD_ARG
    assert raw(lib, "rphys_body_set_velocity", w.h, sid, byref(rp.vel((float("inf"), 0, 0)))) == rp.RPHYS_ERR_BAD_ARG
    assert raw(lib, "rphys_body_apply_impulse", w.h, sid, rp.Vec3(float("nan"), 0, 0)) == rp.RPHYS_ERR_BAD_ARG


def case_last_error_thread_local_and_copy(lib):
    # tests.rs:1390-1414, 1450-1463, 1498-1513
    w = mk_world(lib)
    pose = rp.Isometry()
    assert raw(lib, "rphys_body_get_pose", w.h, 99, byref(pose)) == rp.RPHYS_ERR_INVALID_ID
    msg = lib.dll.rphys_last_error_message()
    assert msg and b"out of range" in msg
    seen = {}

    def other():
        seen["msg"] = lib.dll.rphys_last_error_message()

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert seen["msg"] is None
    n = c_uint32(0)
    buf = ctypes.create_string_buffer(8)
    assert raw(lib, "rphys_last_error_copy", buf, 8, byref(n)) == rp.RPHYS_OK
    assert n.value == len(msg) and buf.value == msg[:7]
    w.step(DT)
    assert lib.dll.rphys_last_error_message() is None


def case_apply_impulse_changes_velocity(lib):
    # tests.rs:891-919
    w = mk_world(lib)
    sid = w.add_sphere((0, 5, 0), 0.5)
    w.apply_impulse(sid, (1.0, 0, 0))
    v, _ = w.velocity(sid)
    assert v[0] > 0.0


# ------------------------------------------------------------------ determinism and rollback
def case_hash_matches_between_two_worlds(lib):
    # tests.rs:337-373 and 1242-1284 (a sphere dropped on a ground box at 120 Hz)
    a, b = mk_world(lib), mk_world(lib)
    for w in (a, b):
        g = c_uint32(0)
        w.c("rphys_add_box_body", byref(box_desc((0, -0.5, 0), (50, 0.5, 50), dynamic=False, mass=0.0)), byref(g))
        w.add_sphere((0, 5, 0), 0.5)
    for _ in range(240):
        assert a.step_hash(1.0 / 120.0) == b.step_hash(1.0 / 120.0)


def rollback_scene(lib):
    # tests.rs:1616-1638
    w = mk_world(lib)
    g = c_uint32(0)
    w.c("rphys_add_box_body", byref(box_desc((0, -0.5, 0), (50, 0.5, 50), dynamic=False, mass=0.0)), byref(g))
    top = 0
    for i in range(3):
        top = c_uint32(0)
        w.c("rphys_add_box_body", byref(box_desc((0, 0.1 + 0.205 * i, 0), (0.2, 0.1, 0.2), mass=5.0)), byref(top))
        top = top.value
    d = c_uint32(0)
    w.c("rphys_add_box_body", byref(box_desc((3, 4, 0), (0.2, 0.2, 0.2), mass=2.0)), byref(d))
    return w, top


def case_rollback_replays(lib, settle, expect_asleep):
    # tests.rs:1652-1684
    w, top = rollback_scene(lib)
    for _ in range(settle):
        w.step_hash(DT)
    st = w.stats()
    assert st["warm_entries"] > 0
    assert (st["sleeping"] > 0) == expect_asleep, st["sleeping"]
    snap = w.snapshot()
    w.apply_impulse(top, (0.3, 0, 0))
    first = [w.step_hash(DT) for _ in range(90)]
    w.restore(snap)
    w.apply_impulse(top, (0.3, 0, 0))
    again = [w.step_hash(DT) for _ in range(90)]
    w.free_snapshot(snap)
    for k, (x, y) in enumerate(zip(first, again)):
        assert x == y, f"step {k + 1} after the restore differs"


def case_rollback_restores_exact_hash(lib):
    # at_rest_test.rs:198-228 (carried_state_restores_exactly): a restore gives back the same hash
    w, _ = rollback_scene(lib)
    for _ in range(40):
        w.step(DT)
    h0 = w.hash()
    snap = w.snapshot()
    for _ in range(10):
        w.step(DT)
    assert w.hash() != h0
    w.restore(snap)
    assert w.hash() == h0
    w.free_snapshot(snap)


def case_exact_restore_replays_rotated_bodies(lib):
    # rphys_ext_snapshot_restore_exact (a World clone): a yawed box pile replays bit for bit
    w = lib.world(64, 64)
    dt, _ = scenes.box_drop(rp, w, n_side=3)
    for _ in range(45):
        w.step(dt)
    snap = w.snapshot()
    first = [w.step_hash(dt) for _ in range(20)]
    w.restore_exact(snap)
    again = [w.step_hash(dt) for _ in range(20)]
    w.free_snapshot(snap)
    assert first == again


def case_teleport_drops_only_its_warm_entries(lib):
    # at_rest_test.rs:230-248
    w, top = rollback_scene(lib)
    for _ in range(30):
        w.step(DT)
    before = w.stats()["warm_entries"]
    p, q = w.pose(4)
    w.c("rphys_body_set_pose", 4, byref(rp.iso(p[0] + 10.0, p[1], p[2], q=q)))  # the dropped box
    after = w.stats()["warm_entries"]
    assert 0 < after <= before


# ------------------------------------------------------------------ acceptance (contact_resting_test.rs, at_rest_test.rs)
def ground_world(lib, cap=16, material=6):
    w = lib.world(cap, cap)
    w.add_bodies([rp.BodyDescEx(rp.iso(0, -0.5, 0), rp.vel(), rp.SHAPE_BOX, (50, 0.5, 50), 0, 0, material, 1)])
    return w


def case_shapes_rest_on_ground(lib):
    # contact_resting_test.rs:30-46 (Rubber bodies on a Concrete ground box, sleep disabled)
    for shape, dims, half_y in ((rp.SHAPE_SPHERE, (0.1, 0, 0), 0.1), (rp.SHAPE_CAPSULE, (0.1, 0.1, 0), 0.2),
                                (rp.SHAPE_BOX, (0.1, 0.1, 0.1), 0.1)):
        for mass in (1.0, 80.0):
            w = ground_world(lib)
            dens = mass / (8 * 0.1 * half_y * 0.1)
            bid = w.add_bodies([rp.BodyDescEx(rp.iso(0, half_y + 0.2, 0), rp.vel(), shape, dims, dens, 1, 2, 0)])
            for _ in range(180):
                w.step(DT)
            y = w.pose(bid)[0][1]
            assert abs(y - half_y) < 0.012, (shape, mass, y)


def case_tilted_box_settles_flat(lib):
    # contact_resting_test.rs:49-61
    w = ground_world(lib)
    q = (0.0, 0.0, math.sin(0.3), math.cos(0.3))
    bid = w.add_bodies([rp.BodyDescEx(rp.iso(0, 0.25, 0, q=q), rp.vel(), rp.SHAPE_BOX, (0.1, 0.1, 0.1), 2.0 / 0.008, 1, 2, 0)])
    for _ in range(300):
        w.step(DT)
    p, r = w.pose(bid)
    x, y, z, ww = r
    # |axis.y| of the box's three axes (rotation matrix row 1)
    ys = [abs(2 * (x * y + ww * z)), abs(1 - 2 * (x * x + z * z)), abs(2 * (y * z - ww * x))]
    assert max(ys) > 0.99 and abs(p[1] - 0.1) < 0.012


def case_stacked_boxes_hold(lib):
    # contact_resting_test.rs:63-74 (30 s kept awake)
    w = ground_world(lib)
    dens = 5.0 / (8 * 0.2 * 0.1 * 0.2)
    ids = [w.add_bodies([rp.BodyDescEx(rp.iso(0, 0.1 + 0.2 * i + 0.01 * i, 0), rp.vel(), rp.SHAPE_BOX, (0.2, 0.1, 0.2),
                                       dens, 1, 2, 0)]) for i in range(3)]
    for _ in range(1800):
        w.step(DT)
    for i, b in enumerate(ids):
        p = w.pose(b)[0]
        assert abs(p[1] - (0.1 + 0.2 * i)) < 0.03 and abs(p[0]) < 0.02 and abs(p[2]) < 0.02


def case_box_rests_on_heightfield(lib):
    # at_rest_test.rs:300-316: a box resting flat on a flat HeightField stays put
    w = lib.world(16, 16)
    h = np.zeros((16, 16), dtype=np.float32)
    w.set_heightfield(h, 16, 16, 1.0, 1.0, -8.0, -8.0, material=4)
    bid = w.add_bodies([rp.BodyDescEx(rp.iso(0.3, 0.21, 0.2), rp.vel(), rp.SHAPE_BOX, (0.2, 0.2, 0.2), 500.0, 1, 0, 0)])
    for _ in range(240):
        w.step(DT)
    p, q = w.pose(bid)
    assert abs(p[1] - 0.2) < 0.012 and abs(p[0] - 0.3) < 0.02 and abs(p[2] - 0.2) < 0.02
    assert w.stats()["contacts"] >= 3
