"""Joints on the GPU: the reference's joint acceptance cases, and tick-by-tick bit parity with the CPU
oracle on jointed scenes (pendulum chains, ragdolls on a heightfield, sleeping ragdolls hit by
falling boxes, the per-island residual stop, batched worlds, rollback, the allocation-free hash)."""
import numpy as np
import pytest

import joint_cases as J
from conftest import rp, scenes
from test_gpu_parity import run_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", [n for n in dir(J) if n.startswith("case_")])
def test_case(gpu, name):
    getattr(J, name)(gpu)


def _chain(rp_, w, n=6, hz=62.5):
    """A pinned chain of rods: ball joints and limited hinges alternating, released horizontal."""
    w.set_gravity((0.0, -9.81, 0.0))
    pos = [(0.0, 12.0, 0.0)] + [(0.5 + 1.0 * k, 12.0, 0.0) for k in range(n)]
    he = [(0.01, 0.01, 0.01)] + [(0.5, 0.04, 0.04)] * n
    d = rp_.desc_array(np.array(pos), np.tile([0.0, 0.0, 0.0, 1.0], (n + 1, 1)), np.array(he), rp_.SHAPE_BOX,
                       np.array([1.0] + [800.0] * n), np.array([0] + [1] * n, dtype=np.uint32))
    first = w.add_bodies_array(d)
    joints = []
    for k in range(n):
        fa = ((0.0, 0.0, 0.0), (0, 0, 0, 1)) if k == 0 else ((0.5, 0.0, 0.0), (0, 0, 0, 1))
        joints.append((rp_.JOINT_BALL if k % 2 == 0 else rp_.JOINT_HINGE, first + k, first + k + 1, fa,
                       ((-0.5, 0.0, 0.0), (0, 0, 0, 1)), 2))
    j0 = w.add_joints(joints)
    for k in range(n):
        if k % 2:
            w.set_joint_limit(j0 + k, True, 2, -1.2, 0.3)
        else:
            w.set_joint_limit(j0 + k, True, 1, -0.6, 0.6)
    return 1.0 / hz, n + 1


def _d6_chain(rp_, w, hz=120.0):
    """A pinned chain of six rods, one D6 feature per joint: a damped torsional spring (XPBD
    Kelvin-Voigt row), a velocity motor, a translational spring with viscous damping, a limited
    position drive, a ball joint with damping and friction on every axis, a limited axis with a
    velocity drive; boxes dropped onto the chain add contacts on jointed bodies."""
    w.set_gravity((0.0, -9.81, 0.0))
    n = 6
    pos = [(0.0, 6.0, 0.0)] + [(0.5 + 1.0 * k, 6.0, 0.0) for k in range(n)]
    he = [(0.01, 0.01, 0.01)] + [(0.5, 0.06, 0.06)] * n
    d = rp_.desc_array(np.array(pos), np.tile([0.0, 0.0, 0.0, 1.0], (n + 1, 1)), np.array(he), rp_.SHAPE_BOX,
                       np.array([1.0] + [600.0] * n), np.array([0] + [1] * n, dtype=np.uint32), sleep_allowed=0)
    first = w.add_bodies_array(d)
    kinds = [rp_.JOINT_D6, rp_.JOINT_HINGE, rp_.JOINT_D6, rp_.JOINT_HINGE, rp_.JOINT_BALL, rp_.JOINT_D6]
    joints = []
    for k in range(n):
        fa = ((0.0, 0.0, 0.0), (0, 0, 0, 1)) if k == 0 else ((0.5, 0.0, 0.0), (0, 0, 0, 1))
        joints.append((kinds[k], first + k, first + k + 1, fa, ((-0.5, 0.0, 0.0), (0, 0, 0, 1)), 2))
    j = w.add_joints(joints)
    w.set_joint_axis(j, True, 2, True, 0.02)
    w.set_joint_damping(j, True, 2, 0.5, 0.0)
    w.set_joint_drive(j + 1, True, 2, 1.5, max_impulse=40.0, velocity=True)
    w.set_joint_damping(j + 1, True, 0, 0.2, 0.1)
    w.set_joint_axis(j + 2, False, 0, True, 2.0e-4)
    w.set_joint_damping(j + 2, False, 0, 3.0, 0.0)
    w.set_joint_damping(j + 2, True, 1, 0.0, 0.3)
    w.set_joint_limit(j + 3, True, 2, -1.0, 0.6)
    w.set_joint_drive(j + 3, True, 2, 0.4, max_impulse=1000.0)
    for ax in range(3):
        w.set_joint_damping(j + 4, True, ax, 0.25, 0.05)
    w.set_joint_limit(j + 5, True, 1, -0.3, 0.3)
    w.set_joint_drive(j + 5, True, 1, -0.8, max_impulse=5.0, velocity=True)
    w.set_joint_axis(j + 5, True, 0, False)
    g = rp_.desc_array(np.array([[3.0, -0.5, 0.0]]), np.array([[0.0, 0.0, 0.0, 1.0]]), np.array([[20.0, 0.5, 20.0]]),
                       rp_.SHAPE_BOX, np.array([0.0]), np.array([0], dtype=np.uint32))
    w.add_bodies_array(g)
    rng = np.random.default_rng(9)
    m = 10
    bp = np.column_stack([rng.uniform(0.5, 6.0, m), rng.uniform(8.0, 11.0, m), rng.uniform(-0.3, 0.3, m)])
    bd = rp_.desc_array(bp, np.tile([0.0, 0.0, 0.0, 1.0], (m, 1)), np.full((m, 3), 0.2), rp_.SHAPE_BOX,
                        np.full(m, 500.0), np.ones(m, dtype=np.uint32))
    w.add_bodies_array(bd)
    return 1.0 / hz, w.num_bodies()


def _distance_scene(rp_, w, hz=120.0):
    """Distance joints of every kind under falling boxes: a rigid centre-to-centre rod, a sprung
    one, an anchored rigid rod (torque through its lever arms), an anchored damped spring, and a
    chain mixing them with a ball joint."""
    w.set_gravity((0.0, -9.81, 0.0))
    pins = [(-6.0, 8.0, 0.0), (-3.0, 8.0, 0.0), (0.0, 8.0, 0.0), (3.0, 8.0, 0.0), (6.0, 8.0, 0.0)]
    d = rp_.desc_array(np.array(pins), np.tile([0.0, 0.0, 0.0, 1.0], (5, 1)), np.full((5, 3), 0.02), rp_.SHAPE_BOX,
                       np.ones(5), np.zeros(5, dtype=np.uint32))
    p0 = w.add_bodies_array(d)
    rng = np.random.default_rng(3)
    bobs = []
    for k in range(5):
        x, y, z = pins[k]
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        bd = rp_.desc_array(np.array([[x + 0.6, y - 0.8, 0.3]]), q[None, :], np.array([[0.15, 0.1, 0.2]]), rp_.SHAPE_BOX,
                            np.array([600.0]), np.ones(1, dtype=np.uint32), sleep_allowed=0,
                            lin=np.array([[0.0, 0.0, 1.0]]), ang=np.array([[0.5, -1.0, 1.5]]))
        bobs.append(w.add_bodies_array(bd))
    w.add_distance_joints([
        (p0, bobs[0], (0, 0, 0), (0, 0, 0), 1.0, 0.0, 0.0),
        (p0 + 1, bobs[1], (0, 0, 0), (0, 0, 0), 0.9, 4.0e-3, 0.0),
        (p0 + 2, bobs[2], (0, 0, 0), (0.1, 0.05, -0.1), 1.1, 0.0, 0.0),
        (p0 + 3, bobs[3], (0.0, -0.01, 0.0), (-0.1, 0.1, 0.0), 0.8, 2.0e-3, 3.0),
        (p0 + 4, bobs[4], (0, 0, 0), (0, 0, 0), 1.0, 0.0, 0.0),
    ])
    # a second link below the last bob: a ball joint then a sprung rod
    bd = rp_.desc_array(np.array([[6.6, 6.2, 0.3], [6.6, 5.0, 0.3]]), np.tile([0.0, 0.0, 0.0, 1.0], (2, 1)),
                        np.full((2, 3), 0.12), rp_.SHAPE_BOX, np.full(2, 700.0), np.ones(2, dtype=np.uint32))
    c0 = w.add_bodies_array(bd)
    w.add_joints([(rp_.JOINT_BALL, bobs[4], c0, ((0.0, -0.3, 0.0), (0, 0, 0, 1)), ((0.0, 0.3, 0.0), (0, 0, 0, 1)), 0)])
    w.add_distance_joints([(c0, c0 + 1, (0, -0.1, 0), (0, 0.1, 0), 1.0, 1.0e-3, 0.0)])
    g = rp_.desc_array(np.array([[0.0, -0.5, 0.0]]), np.array([[0.0, 0.0, 0.0, 1.0]]), np.array([[20.0, 0.5, 20.0]]),
                       rp_.SHAPE_BOX, np.array([0.0]), np.array([0], dtype=np.uint32))
    w.add_bodies_array(g)
    m = 8
    bp = np.column_stack([rng.uniform(-6.0, 6.0, m), rng.uniform(9.0, 12.0, m), rng.uniform(-0.2, 0.6, m)])
    bd = rp_.desc_array(bp, np.tile([0.0, 0.0, 0.0, 1.0], (m, 1)), np.full((m, 3), 0.2), rp_.SHAPE_BOX,
                        np.full(m, 500.0), np.ones(m, dtype=np.uint32))
    w.add_bodies_array(bd)
    return 1.0 / hz, w.num_bodies()


def test_distance_joints(oracle, gpu):
    run_pair(oracle, gpu, {"cap": (32, 32), "fn": lambda rp_, w: _distance_scene(rp_, w)}, 600)


def test_distance_joints_60hz(oracle, gpu):
    run_pair(oracle, gpu, {"cap": (32, 32), "fn": lambda rp_, w: _distance_scene(rp_, w, 60.0)}, 300)


def test_d6_feature_chain(oracle, gpu):
    run_pair(oracle, gpu, {"cap": (32, 32), "fn": lambda rp_, w: _d6_chain(rp_, w)}, 600)


def test_d6_feature_chain_60hz(oracle, gpu):
    run_pair(oracle, gpu, {"cap": (32, 32), "fn": lambda rp_, w: _d6_chain(rp_, w, 60.0)}, 300)


def _ragdolls(n, **kw):
    def build(rp_, w):
        dt, nb, _ = scenes.ragdolls(rp_, w, n_ragdolls=n, **kw)
        return dt, nb
    return build


def test_pendulum_chain(oracle, gpu):
    build = {"cap": (16, 16), "fn": lambda rp_, w: _chain(rp_, w)}
    run_pair(oracle, gpu, build, 400)


def test_ragdolls_on_terrain(oracle, gpu):
    build = {"cap": (1024, 1024), "fn": _ragdolls(10)}
    run_pair(oracle, gpu, build, 240, check_every=4)


def test_ragdolls_with_muscles_on_terrain(oracle, gpu):
    build = {"cap": (1024, 1024), "fn": _ragdolls(10, muscles=True)}
    run_pair(oracle, gpu, build, 240, check_every=4)


def test_ragdolls_residual_mode(oracle, gpu):
    def build(rp_, w):
        out = _ragdolls(8)(rp_, w)
        w.set_residual_mode(1e-4, 96)
        return out
    run_pair(oracle, gpu, {"cap": (1024, 1024), "fn": build}, 200, check_every=4)


def test_sleeping_ragdolls_hit_by_boxes(oracle, gpu):
    """Ragdolls piled in a small area settle and fall asleep limb by limb; boxes dropped on them later
    meet sleeping limbs whose joints still tie them to awake ones."""
    def build(rp_, w):
        dt, nb, _ = scenes.ragdolls(rp_, w, n_ragdolls=12, flat_area=8.0)
        return dt, nb
    wo, wg = oracle.world(2048, 2048), gpu.world(2048, 2048)
    dt, _ = build(rp, wo)
    build(rp, wg)
    asleep = 0
    for t in range(480):
        wo.step(dt); wg.step(dt)
        if t % 20 == 19:
            assert wo.hash() == wg.hash(), f"tick {t}: hash differs"
        asleep = max(asleep, wo.stats()["sleeping"])
    assert asleep > 0, "nothing fell asleep: the case does not exercise sleeping jointed bodies"
    rng = np.random.default_rng(4)
    n = 24
    pos = np.column_stack([rng.uniform(-3, 3, n), rng.uniform(3, 6, n), rng.uniform(-3, 3, n)])
    d = rp.desc_array(pos, np.tile([0.0, 0.0, 0.0, 1.0], (n, 1)), np.full((n, 3), 0.3), rp.SHAPE_BOX,
                      np.full(n, 2000.0), np.ones(n, dtype=np.uint32))
    wo.add_bodies_array(d); wg.add_bodies_array(d)
    for t in range(300):
        wo.step(dt); wg.step(dt)
        so, sg = wo.body_states(), wg.body_states()
        assert np.array_equal(so.view(np.uint32), sg.view(np.uint32)), f"tick {t}: body bits differ"
        assert wo.hash() == wg.hash(), f"tick {t}: hash differs"
        for k in ("contacts", "islands", "levels", "max_batch", "sleeping", "rows_scheduled", "row_sweeps"):
            assert wo.stats()[k] == wg.stats()[k], f"tick {t}: stat {k}"


def test_batched_ragdoll_worlds(oracle, gpu):
    """Worlds of ragdolls in one batched device world: each world's hash equals the oracle running
    that world alone."""
    k_worlds, per = 6, 3
    h, origin = scenes.heightfield(64, 1.0, 5)
    wg = gpu.world(4096, 4096)
    wg.set_heightfield(h, 64, 64, 1.0, 1.0, origin, origin, material=4)
    singles = []
    for k in range(k_worlds):
        first = wg.num_bodies() + 1
        bd, jd, ld = scenes.ragdoll_arrays(rp, per, 100 + k, 40.0, base_id=first, y0=float(h.max()) + 1.0)
        wg.add_world(bd)
        j0 = wg.add_joint_array(jd)
        ld[:, 0].view(np.uint32)[:] += j0
        wg.set_joint_limit_array(ld)
        bo, jo, lo = scenes.ragdoll_arrays(rp, per, 100 + k, 40.0, base_id=1, y0=float(h.max()) + 1.0)
        wo = oracle.world(len(bo), len(bo))  # a world's hash covers its capacity: the batch's is its body count
        wo.set_heightfield(h, 64, 64, 1.0, 1.0, origin, origin, material=4)
        wo.add_bodies_array(bo)
        wo.add_joint_array(jo)
        wo.set_joint_limit_array(lo)
        singles.append(wo)
    for w in [wg] + singles:
        w.set_pair_props(0, 0, 0.6, 0.5, 0.0, 0.08)
        w.set_pair_props(0, 4, 0.883176, 0.724569, 0.0, 0.1)
        w.set_iterations(24, 24)
    dt = 1.0 / 120.0
    for t in range(180):
        wg.step(dt)
        for wo in singles:
            wo.step(dt)
        if t % 30 == 29:
            hs = wg.world_hashes()
            for k, wo in enumerate(singles):
                assert hs[k] == wo.hash(), f"tick {t}: world {k} hash differs"


def test_ragdoll_rollback_replays_exactly(gpu):
    w = gpu.world(1024, 1024)
    dt, _, _ = scenes.ragdolls(rp, w, n_ragdolls=8)
    for _ in range(60):
        w.step(dt)
    snap = w.snapshot()
    for _ in range(30):
        w.step(dt)
    h1, s1 = w.hash(), w.body_states()
    w.restore_exact(snap)
    for _ in range(30):
        w.step(dt)
    assert w.hash() == h1
    assert np.array_equal(w.body_states().view(np.uint32), s1.view(np.uint32))
    w.free_snapshot(snap)


def test_noalloc_hash_with_joints(gpu):
    w = gpu.world(1024, 1024)
    dt, _, _ = scenes.ragdolls(rp, w, n_ragdolls=6)
    for _ in range(40):
        w.step(dt)
    assert w.hash_noalloc() == w.hash()
