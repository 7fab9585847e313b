"""Joint acceptance cases over any library exporting the C ABI (the CPU oracle in
tests/test_oracle_joints.py, the CUDA library in tests/test_gpu_joints.py). Restated from the
reference's riftphys-world/tests/joint_energy_test.rs:46-219 (SHAKE energy behaviour, limits,
replay) and hinge_angle_test.rs:14-58 (hinge limits in radians), with the same bodies, rates and
tolerances; the pin bodies carry a small collider here (the FFI gives every body one), which never
touches the jointed rods."""
import math

import numpy as np

from conftest import rp

G = 9.81


def _world(lib, cap=8):
    w = lib.world(cap, cap)
    w.set_gravity((0.0, -G, 0.0))
    return w


def _body(w, pos, he, density, dynamic=True, rot=(0.0, 0.0, 0.0, 1.0), lin=(0.0, 0.0, 0.0), ang=(0.0, 0.0, 0.0)):
    d = rp.desc_array(np.array([pos]), np.array([rot]), np.array([he]), rp.SHAPE_BOX, np.array([density]),
                      np.array([1 if dynamic else 0], dtype=np.uint32), lin=np.array([lin]), ang=np.array([ang]))
    return w.add_bodies_array(d)


def _box_mass(he, rho):
    m = 8.0 * he[0] * he[1] * he[2] * rho
    return m, np.diag([m / 3.0 * (he[1] ** 2 + he[2] ** 2), m / 3.0 * (he[0] ** 2 + he[2] ** 2),
                       m / 3.0 * (he[0] ** 2 + he[1] ** 2)])


def _rotm(q):
    x, y, z, w_ = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w_ * z), 2 * (x * z + w_ * y)],
                     [2 * (x * y + w_ * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w_ * x)],
                     [2 * (x * z - w_ * y), 2 * (y * z + w_ * x), 1 - 2 * (x * x + y * y)]])


def _energy(w, bid, m, inertia, y0):
    (p, q), (l, a) = w.pose(bid), w.velocity(bid)
    r = _rotm(q)
    iw = r @ inertia @ r.T
    a = np.array(a)
    return m * G * (p[1] - y0) + 0.5 * m * float(np.dot(l, l)) + 0.5 * float(a @ iw @ a)


PIN = (0.01, 0.01, 0.01)
ROD = (0.5, 0.025, 0.025)
ID = ((0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 1.0))


def _hinge(w, a, b, fa_pos, fb_pos, axis=2):
    return w.add_joints([(rp.JOINT_HINGE, a, b, (fa_pos, (0, 0, 0, 1)), (fb_pos, (0, 0, 0, 1)), axis)])


def _cube_pendulum(lib):
    # an 80 kg, 2 m cube on a 5 m arm about z, released horizontal (joint_energy_test.rs:46-54)
    w = _world(lib)
    p = _body(w, (0.0, 20.0, 0.0), PIN, 1.0, dynamic=False)
    bob = _body(w, (5.0, 20.0, 0.0), (1.0, 1.0, 1.0), 10.0)
    _hinge(w, p, bob, (0.0, 0.0, 0.0), (-5.0, 0.0, 0.0))
    m, inertia = _box_mass((1.0, 1.0, 1.0), 10.0)
    return w, bob, m, inertia


def case_hinge_pendulum_keeps_its_energy(lib):
    """joint_energy_test.rs:72-79: swing energy within 2% (5 s at 62.5 and 240 Hz)."""
    for hz, secs, tol in ((62.5, 5.0, 0.02), (240.0, 5.0, 0.02)):
        w, bob, m, inertia = _cube_pendulum(lib)
        dt = 1.0 / hz
        w.step(dt)
        e0 = _energy(w, bob, m, inertia, 15.0)
        lo = hi = 1.0
        for _ in range(int(secs * hz)):
            w.step(dt)
            r = _energy(w, bob, m, inertia, 15.0) / e0
            lo, hi = min(lo, r), max(hi, r)
        assert lo > 1.0 - tol and hi < 1.0 + tol, f"{hz} Hz: swing energy ranged {lo:.4f}..{hi:.4f}"
        w.close()


def case_ball_joint_spherical_pendulum(lib):
    """joint_energy_test.rs:154-182: a 1 m rod on a ball joint, released 60 degrees out spinning at
    3 rad/s about the vertical: energy and vertical angular momentum conserved (62.5 Hz: 5%, 2%)."""
    hz, e_tol = 62.5, 0.05
    w = _world(lib)
    pivot = np.array([0.0, 10.0, 0.0])
    p = _body(w, tuple(pivot), PIN, 1.0, dynamic=False)
    d = np.array([math.sin(math.radians(60)), -math.cos(math.radians(60)), 0.0])
    centre = pivot + 0.5 * d
    spin = np.array([0.0, 3.0, 0.0])
    th = math.atan2(d[1], d[0])  # rotation about z taking x to d
    q = (0.0, 0.0, math.sin(0.5 * th), math.cos(0.5 * th))
    r = _body(w, tuple(centre), ROD, 1000.0, rot=q, lin=tuple(np.cross(spin, centre - pivot)), ang=tuple(spin))
    w.add_joints([(rp.JOINT_BALL, p, r, ID, ((-0.5, 0.0, 0.0), (0, 0, 0, 1)), 0)])
    m, inertia = _box_mass(ROD, 1000.0)

    def l_y():
        (ps, qq), (lv, av) = w.pose(r), w.velocity(r)
        rm = _rotm(qq)
        return (np.cross(np.array(ps) - pivot, np.array(lv) * m) + (rm @ inertia @ rm.T) @ np.array(av))[1]

    dt = 1.0 / hz
    w.step(dt)
    e0, l0 = _energy(w, r, m, inertia, 9.5), l_y()
    e_err = l_err = 0.0
    for _ in range(int(10.0 * hz)):
        w.step(dt)
        e_err = max(e_err, abs(_energy(w, r, m, inertia, 9.5) / e0 - 1.0))
        l_err = max(l_err, abs(l_y() / l0 - 1.0))
    assert e_err < e_tol, f"spherical pendulum energy drifted {100 * e_err:.2f}%"
    assert l_err < 0.02, f"vertical angular momentum drifted {100 * l_err:.2f}%"
    w.close()


def case_hinge_limit_still_absorbs_energy(lib):
    """joint_energy_test.rs:187-207: a rod swinging into a stop at -1.8 rad keeps < 50% of its swing
    energy, and never gains more than 5%."""
    for hz in (62.5, 240.0):
        w = _world(lib)
        p = _body(w, (0.0, 10.0, 0.0), PIN, 1.0, dynamic=False)
        a = _body(w, (0.5, 10.0, 0.0), ROD, 1000.0)
        j = _hinge(w, p, a, (0.0, 0.0, 0.0), (-0.5, 0.0, 0.0))
        w.set_joint_limit(j, True, 2, -1.8, 0.1)
        m, inertia = _box_mass(ROD, 1000.0)
        dt = 1.0 / hz
        w.step(dt)
        e0 = _energy(w, a, m, inertia, 9.5)
        peak = 1.0
        for _ in range(int(5.0 * hz)):
            w.step(dt)
            peak = max(peak, _energy(w, a, m, inertia, 9.5) / e0)
        kept = _energy(w, a, m, inertia, 9.5) / e0
        assert kept < 0.5 and peak < 1.05, f"{hz} Hz: kept {kept:.3f} of the swing energy (peak {peak:.3f})"
        w.close()


def _rod_angle(q):
    # to_axis_angle, signed by the axis' z (hinge_angle_test.rs:23-26)
    x, y, z, w_ = q
    s = math.sqrt(x * x + y * y + z * z)
    a = 2.0 * math.atan2(s, w_)
    if abs(a) < 1e-6 or s == 0.0:
        return 0.0
    return a * math.copysign(1.0, z / s)


def _swing(lib, lo, hi, secs):
    w = _world(lib, 4)
    p = _body(w, (0.0, 10.0, 0.0), PIN, 1.0, dynamic=False)
    r = _body(w, (0.5, 10.0, 0.0), ROD, 1000.0)
    j = _hinge(w, p, r, (0.0, 0.0, 0.0), (-0.5, 0.0, 0.0))
    w.set_joint_limit(j, True, 2, lo, hi)
    furthest = 0.0
    for _ in range(int(secs * 240.0)):
        w.step(1.0 / 240.0)
        a = _rod_angle(w.pose(r)[1])
        if abs(a) > abs(furthest):
            furthest = a
    rest = _rod_angle(w.pose(r)[1])
    w.close()
    return math.degrees(furthest), math.degrees(rest)


def case_hinge_rests_on_a_limit_in_radians(lib):
    """hinge_angle_test.rs:44-49: a stop at -1 rad: the rod falls onto it and rests there."""
    furthest, rest = _swing(lib, -1.0, 1.0, 5.0)
    stop = math.degrees(-1.0)
    assert abs(rest - stop) < 0.5, f"rested at {rest:.2f} deg, stop at {stop:.2f}"
    assert furthest > stop - 1.0, f"overshot to {furthest:.2f} deg"


def case_hinge_limit_beyond_two_radians_holds(lib):
    """hinge_angle_test.rs:54-58: a stop at -2.2 rad, past the bottom of the swing, is reached and held."""
    furthest, _ = _swing(lib, -2.2, 0.1, 3.0)
    stop = math.degrees(-2.2)
    assert stop - 1.0 < furthest < stop + 1.0, f"furthest {furthest:.2f} deg, stop at {stop:.2f}"


def case_shake_replays_bit_exactly(lib):
    """joint_energy_test.rs:210-221: two runs of the cube pendulum end in identical bits."""
    out = []
    for _ in range(2):
        w, bob, _, _ = _cube_pendulum(lib)
        for _ in range(300):
            w.step(1.0 / 62.5)
        out.append((w.pose(bob), w.velocity(bob), w.hash()))
        w.close()
    assert out[0] == out[1]


def case_jointed_bodies_do_not_collide(lib):
    """step.rs:85-102: two overlapping boxes joined by a ball joint make no contact; unjoined they do."""
    for joined in (True, False):
        w = lib.world(4, 4)
        a = _body(w, (0.0, 5.0, 0.0), (0.5, 0.5, 0.5), 1000.0)
        b = _body(w, (0.6, 5.0, 0.0), (0.5, 0.5, 0.5), 1000.0)
        if joined:
            w.add_joints([(rp.JOINT_BALL, a, b, ((0.3, 0.0, 0.0), (0, 0, 0, 1)), ((-0.3, 0.0, 0.0), (0, 0, 0, 1)), 0)])
        w.step(1.0 / 60.0)
        n = w.stats()["contacts"]
        assert (n == 0) if joined else (n > 0), f"joined={joined}: {n} contacts"
        w.close()


def case_joint_api_errors(lib):
    """Argument checks of the joint entry points (ids as everywhere in the C ABI)."""
    w = lib.world(4, 4)
    a = _body(w, (0.0, 1.0, 0.0), (0.5, 0.5, 0.5), 1000.0)
    b = _body(w, (2.0, 1.0, 0.0), (0.5, 0.5, 0.5), 1000.0)
    bad = [
        [(rp.JOINT_BALL, a, a, ID, ID, 0)],            # same body
        [(rp.JOINT_BALL, a, 99, ID, ID, 0)],           # no such body
        [(rp.JOINT_HINGE, a, b, ID, ID, 3)],           # hinge axis out of range
        [(7, a, b, ID, ID, 0)],                        # unknown kind
        [(rp.JOINT_BALL, a, b, ((float("nan"), 0, 0), (0, 0, 0, 1)), ID, 0)],
    ]
    for j in bad:
        try:
            w.add_joints(j)
        except rp.RPhysError:
            pass
        else:
            raise AssertionError(f"accepted {j}")
    assert w.num_joints() == 0
    j = w.add_joints([(rp.JOINT_BALL, a, b, ID, ID, 0), (rp.JOINT_HINGE, a, b, ID, ID, 1)])
    assert j == 0 and w.num_joints() == 2
    for args in ((5, True, 1, -1.0, 1.0), (0, True, 3, -1.0, 1.0), (0, True, 1, 1.0, -1.0), (0, False, 0, 0.0, float("inf"))):
        try:
            w.set_joint_limit(*args)
        except rp.RPhysError:
            pass
        else:
            raise AssertionError(f"accepted limit {args}")
    w.set_joint_limit(0, True, 1, -0.5, 0.5)
    w.set_joint_limit(0, True, 1)  # cleared
    w.close()
