"""Joint acceptance cases over any library exporting the C ABI (the CPU oracle in
tests/test_oracle_joints.py, the CUDA library in tests/test_gpu_joints.py). Restated from the
reference's riftphys-world/tests: joint_energy_test.rs:46-219 (SHAKE energy behaviour, limits,
replay), hinge_angle_test.rs:14-58 (hinge limits in radians), joint_damping_test.rs (viscous damping
and Coulomb friction rows), compliant_joint_test.rs:20-75, 134-170 (torsional springs and sprung
hinges), joint_conditioning_test.rs:22-66 (position drive, SHAKE projection) and
world_robotics_test.rs:75-135 (velocity motor), distance joints from compliant_joint_test.rs:77-131
and the golden bits of distance_bits_test.rs, with the same bodies, rates and tolerances; the pin
bodies carry a small collider here (the FFI gives every body one), which never touches the jointed
rods (jointed pairs make no contacts)."""
import math

import numpy as np

from conftest import rp

G = 9.81


def _world(lib, cap=8):
    w = lib.world(cap, cap)
    w.set_gravity((0.0, -G, 0.0))
    return w


def _body(w, pos, he, density, dynamic=True, rot=(0.0, 0.0, 0.0, 1.0), lin=(0.0, 0.0, 0.0), ang=(0.0, 0.0, 0.0),
          sleep=True):
    d = rp.desc_array(np.array([pos]), np.array([rot]), np.array([he]), rp.SHAPE_BOX, np.array([density]),
                      np.array([1 if dynamic else 0], dtype=np.uint32), sleep_allowed=1 if sleep else 0,
                      lin=np.array([lin]), ang=np.array([ang]))
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


# ---- viscous damping and Coulomb friction on a hinge (joint_damping_test.rs)
BAR = (0.5, 0.1, 0.1)
BAR_MASS = 2.0
BAR_I = BAR_MASS / 3.0 * (BAR[0] ** 2 + BAR[1] ** 2)  # about z


def _spinner(lib, w0):
    """joint_damping_test.rs:17-25: a 2 kg bar hinged about z through its centre to a static anchor,
    spinning at w0 about z, no gravity, never asleep."""
    w = lib.world(4, 4)
    w.set_gravity((0.0, 0.0, 0.0))
    p = _body(w, (0.0, 0.0, 0.0), PIN, 1.0, dynamic=False)
    b = _body(w, (0.0, 0.0, 0.0), BAR, BAR_MASS / (8.0 * BAR[0] * BAR[1] * BAR[2]), ang=(0.0, 0.0, w0), sleep=False)
    j = _hinge(w, p, b, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    return w, b, j


class _Unwrap:
    """Twist about z, unwrapped step to step (joint_damping_test.rs:28-41)."""

    def __init__(self):
        self.last = self.total = 0.0

    def update(self, q):
        a = 2.0 * math.atan2(q[2], q[3])
        d = a - self.last
        while d > math.pi:
            d -= 2.0 * math.pi
        while d < -math.pi:
            d += 2.0 * math.pi
        self.last = a
        self.total += d
        return self.total


def case_damped_hinge_decays_at_the_closed_form_rate(lib):
    """joint_damping_test.rs:43-66: the implicit damper's decay rate ln(1 + c dt / I) / dt within 0.5%,
    c / I within 2%; the bar stays on its axis."""
    for hz in (60.0, 240.0):
        for rate in (0.5, 2.0):
            w, b, j = _spinner(lib, 3.0)
            w.set_joint_damping(j, True, 2, rate * BAR_I, 0.0)
            t = 2.0
            for _ in range(int(t * hz)):
                w.step(1.0 / hz)
            lin, ang = w.velocity(b)
            measured = math.log(3.0 / ang[2]) / t
            discrete = math.log(1.0 + rate / hz) * hz
            assert abs(measured - discrete) < 0.005 * discrete, f"{hz} Hz, c/I {rate}: rate {measured:.4f}, discrete {discrete:.4f}"
            assert abs(measured - rate) < 0.02 * rate, f"{hz} Hz, c/I {rate}: rate {measured:.4f}"
            assert abs(ang[0]) < 1e-4 and abs(ang[1]) < 1e-4 and np.linalg.norm(lin) < 1e-4, f"off-axis motion {lin} {ang}"
            w.close()


def case_friction_only_with_zero_damping_is_finite(lib):
    """joint_damping_test.rs:68-80: friction without damping is finite; NaN / negative coefficients
    become 0 and act on nothing."""
    w, b, j = _spinner(lib, 3.0)
    w.set_joint_damping(j, True, 2, 0.0, 0.2)
    for _ in range(60):
        w.step(1.0 / 60.0)
    wz = w.velocity(b)[1][2]
    assert math.isfinite(wz) and wz < 3.0, f"w {wz}"
    w.set_joint_damping(j, True, 2, float("nan"), -1.0)
    before = w.velocity(b)[1][2]
    w.step(1.0 / 60.0)
    assert abs(w.velocity(b)[1][2] - before) < 1e-5, "a NaN / negative coefficient acted"
    w.close()


def case_friction_hinge_stops_at_the_closed_form_angle(lib):
    """joint_damping_test.rs:82-99: Coulomb friction tau stops the bar after I w0^2 / (2 tau) (2%) and
    holds it at rest."""
    w0, tau = 3.0, 0.2
    want = BAR_I * w0 * w0 / (2.0 * tau)
    t_stop = BAR_I * w0 / tau
    for hz in (60.0, 240.0):
        w, b, j = _spinner(lib, w0)
        w.set_joint_damping(j, True, 2, 0.0, tau)
        u = _Unwrap()
        angle = 0.0
        for _ in range(int((t_stop + 2.0) * hz)):
            w.step(1.0 / hz)
            angle = u.update(w.pose(b)[1])
        assert abs(angle - want) < 0.02 * want, f"{hz} Hz: stopped after {angle:.4f} rad, want {want:.4f}"
        assert abs(w.velocity(b)[1][2]) < 1e-4, f"{hz} Hz: still turning"
        w.close()


def case_very_stiff_damping_is_stable(lib):
    """joint_damping_test.rs:101-118: c dt / I far above 1 never reverses the spin."""
    for hz in (60.0, 240.0):
        w, b, j = _spinner(lib, 3.0)
        w.set_joint_damping(j, True, 2, 1.0e4 * BAR_I, 0.0)
        last = 3.0
        for _ in range(int(hz)):
            w.step(1.0 / hz)
            wz = w.velocity(b)[1][2]
            assert math.isfinite(wz) and wz >= -1e-6 and wz <= last + 1e-6, f"{hz} Hz: w went {last} -> {wz}"
            last = wz
        assert last < 1e-3, f"{hz} Hz: w still {last}"
        w.close()


def case_damping_on_a_limited_hinge_still_stops_at_the_limit(lib):
    """joint_damping_test.rs:120-131: damping and a limit on one axis: the limit rows still hold."""
    w, b, j = _spinner(lib, 3.0)
    w.set_joint_damping(j, True, 2, 0.05, 0.0)
    w.set_joint_limit(j, True, 2, -0.5, 0.5)
    u = _Unwrap()
    furthest = 0.0
    for _ in range(480):
        w.step(1.0 / 240.0)
        furthest = max(furthest, u.update(w.pose(b)[1]))
    assert furthest < 0.5 + 0.02, f"passed the limit: {furthest:.4f} rad"
    w.close()


# ---- compliant axes (compliant_joint_test.rs)
def _quat_z(a):
    return (0.0, 0.0, math.sin(0.5 * a), math.cos(0.5 * a))


def _rotate(q, v):
    return _rotm(q) @ np.asarray(v, dtype=np.float64)


def _torsion_spring(lib, c, hz, secs):
    """compliant_joint_test.rs:23-53: a 1 m, 2.5 kg rod held out by a torsional spring about z
    (compliance c, rad per N m) on a D6 joint with every other axis rigid, started at its static sag;
    returns the worst departure from the sag, relative to it."""
    w = _world(lib, 4)
    p = _body(w, (0.0, 10.0, 0.0), PIN, 1.0, dynamic=False)
    m = 8.0 * ROD[0] * ROD[1] * ROD[2] * 1000.0
    theta = 0.0
    for _ in range(200):
        theta = np.float32(0.5 * theta + 0.5 * c * m * G * 0.5 * math.cos(theta))
    theta = float(theta)
    q = _quat_z(-theta)
    rod = _body(w, tuple(np.array([0.0, 10.0, 0.0]) + _rotate(q, (0.5, 0.0, 0.0))), ROD, 1000.0, rot=q, sleep=False)
    j = w.add_joints([(rp.JOINT_D6, p, rod, ID, ((-0.5, 0.0, 0.0), (0, 0, 0, 1)), 0)])
    w.set_joint_axis(j, True, 2, True, c)
    worst = 0.0
    for _ in range(int(secs * hz)):
        w.step(1.0 / hz)
        x, y, z, qw = w.pose(rod)[1]
        s2 = 1.0 - qw * qw
        if s2 >= 1e-8:
            ang, az = 2.0 * math.acos(max(-1.0, min(1.0, qw))), z / math.sqrt(s2)
        else:
            ang, az = 0.0, 0.0
        sag = -ang * math.copysign(1.0, az)
        worst = max(worst, abs(sag - theta) / theta)
    w.close()
    return worst


def case_torsional_spring_holds_its_static_sag(lib):
    """compliant_joint_test.rs:55-61: within 3% of the static sag over 10 s (60 and 240 Hz)."""
    for hz in (60.0, 240.0):
        worst = _torsion_spring(lib, 0.008, hz, 10.0)
        assert worst < 0.03, f"{hz} Hz: sag departed {100 * worst:.2f}% from static"


def case_torsional_spring_large_sag_is_in_radians(lib):
    """compliant_joint_test.rs:63-75: a soft spring sagging about 1 rad acts on the angle itself
    (0.25% at 60 Hz, 0.5% at 240 Hz)."""
    for hz, gate in ((60.0, 0.0025), (240.0, 0.005)):
        worst = _torsion_spring(lib, 0.15, hz, 10.0)
        assert worst < gate, f"{hz} Hz: sag departed {100 * worst:.3f}% from static"


def _sprung_hinge_past_90(lib, align_c, hz):
    """compliant_joint_test.rs:134-160: a 1 m rod hinged at its end about z by a spring (c = 0.15),
    started 2.5 rad round and spinning 0.3 rad/s about x, no gravity; the x and y rows at compliance
    align_c and no stored hinge axis. Returns (worst hinge-axis tilt in degrees, worst anchor gap)."""
    w = lib.world(4, 4)
    w.set_gravity((0.0, 0.0, 0.0))
    p = _body(w, (0.0, 10.0, 0.0), PIN, 1.0, dynamic=False)
    q = _quat_z(2.5)
    rod = _body(w, tuple(np.array([0.0, 10.0, 0.0]) + _rotate(q, (0.5, 0.0, 0.0))), ROD, 1000.0, rot=q,
                ang=(0.3, 0.0, 0.0), sleep=False)
    j = w.add_joints([(rp.JOINT_D6, p, rod, ID, ((-0.5, 0.0, 0.0), (0, 0, 0, 1)), 0)])
    w.set_joint_axis(j, True, 0, True, align_c)
    w.set_joint_axis(j, True, 1, True, align_c)
    w.set_joint_axis(j, True, 2, True, 0.15)
    tilt = gap = 0.0
    for _ in range(int(10.0 * hz)):
        w.step(1.0 / hz)
        pos, qq = w.pose(rod)
        z = _rotate(qq, (0.0, 0.0, 1.0))
        tilt = max(tilt, math.degrees(math.acos(max(-1.0, min(1.0, z[2])))))
        gap = max(gap, float(np.linalg.norm(np.array(pos) + _rotate(qq, (-0.5, 0.0, 0.0)) - np.array([0.0, 10.0, 0.0]))))
    w.close()
    return tilt, gap


def case_sprung_hinge_stays_aligned_past_90_degrees(lib):
    """compliant_joint_test.rs:162-172: alignment rows rigid, 1e-9 and 1e-3, the hinge recognised from
    its rows: tilt < 1 degree, gap < 1 mm."""
    for align_c in (0.0, 1.0e-9, 1.0e-3):
        for hz in (60.0, 240.0):
            tilt, gap = _sprung_hinge_past_90(lib, align_c, hz)
            assert tilt < 1.0 and gap < 0.001, f"c {align_c:g}, {hz} Hz: tilt {tilt:.2f} deg, gap {gap:.4f} m"


# ---- drives
def _hinge_angle_z(q):
    x, y, z, qw = q
    if qw < 0.0:
        z, qw = -z, -qw
    return 2.0 * math.atan2(z, qw)


def case_hinge_position_drive_reaches_its_target(lib):
    """joint_conditioning_test.rs:22-66 (the SHAKE projection): a 1 m, 2.5 kg rod hinged at its end
    about z with a rigid position drive to 1 rad holds it within 0.1 degree after 0.1 s, joint apart
    < 1 mm, at 60 / 240 Hz, with and without gravity, 20 and 21 position iterations."""
    target = math.degrees(1.0)
    for hz in (60.0, 240.0):
        for gravity in (0.0, G):
            for pos_iters in (20, 21):
                w = lib.world(4, 4)
                w.set_iterations(20, pos_iters)
                w.set_gravity((0.0, -gravity, 0.0))
                p = _body(w, (0.0, 10.0, 0.0), PIN, 1.0, dynamic=False)
                r = _body(w, (0.5, 10.0, 0.0), ROD, 1000.0)
                j = _hinge(w, p, r, (0.0, 0.0, 0.0), (-0.5, 0.0, 0.0))
                w.set_joint_drive(j, True, 2, 1.0, kp=0.0, kd=0.0, max_impulse=1000.0, velocity=False)
                worst = gap = 0.0
                for k in range(int(hz)):
                    w.step(1.0 / hz)
                    if k / hz >= 0.1:
                        pos, q = w.pose(r)
                        worst = max(worst, abs(math.degrees(_hinge_angle_z(q)) - target))
                        gap = max(gap, float(np.linalg.norm(np.array(pos) + _rotate(q, (-0.5, 0.0, 0.0)) - np.array([0.0, 10.0, 0.0]))))
                assert worst < 0.1, f"{hz} Hz g {gravity} iters {pos_iters}: off target by {worst:.3f} deg"
                assert gap < 0.001, f"{hz} Hz g {gravity} iters {pos_iters}: joint apart by {gap:.4f} m"
                w.close()


def case_hinge_velocity_motor_turns_the_leg(lib):
    """world_robotics_test.rs:75-135: a 0.2 x 1 x 0.2 m leg hanging from a hinge about x, driven by a
    velocity motor at 2 rad/s (max impulse 1000): after 30 ticks of 16 ms it turns at > 1.5 rad/s and
    has swung to z < -0.7, y > 9.3."""
    w = _world(lib, 32)
    p = _body(w, (0.0, 10.0, 0.0), PIN, 1.0, dynamic=False)
    leg = _body(w, (0.0, 9.0, 0.0), (0.1, 0.5, 0.1), 50.0)
    j = w.add_joints([(rp.JOINT_HINGE, p, leg, ID, ((0.0, 1.0, 0.0), (0, 0, 0, 1)), 0)])
    w.set_joint_drive(j, True, 0, 2.0, kp=0.0, kd=5.0, max_impulse=1000.0, velocity=True)
    for _ in range(30):
        w.step(0.016)
    pos, _ = w.pose(leg)
    ang = w.velocity(leg)[1]
    assert ang[0] > 1.5, f"motor at {ang[0]:.3f} rad/s"
    assert pos[2] < -0.7 and pos[1] > 9.3, f"leg at {pos}"
    w.close()


def case_d6_api_errors(lib):
    """Argument checks of the D6 axis, drive and damping entry points."""
    w = lib.world(4, 4)
    a = _body(w, (0.0, 1.0, 0.0), (0.5, 0.5, 0.5), 1000.0)
    b = _body(w, (2.0, 1.0, 0.0), (0.5, 0.5, 0.5), 1000.0)
    j = w.add_joints([(rp.JOINT_D6, a, b, ID, ID, 0)])
    calls = [
        lambda: w.set_joint_axis(5, True, 0, True, 0.0),
        lambda: w.set_joint_axis(j, True, 3, True, 0.0),
        lambda: w.set_joint_axis(j, True, 0, True, -1.0),
        lambda: w.set_joint_axis(j, True, 0, True, float("nan")),
        lambda: w.set_joint_drive(j, True, 3, 1.0),
        lambda: w.set_joint_drive(5, False, 0, 1.0),
        lambda: w.set_joint_drive(j, True, 0, float("inf")),
        lambda: w.set_joint_drive(j, True, 0, 1.0, max_impulse=float("nan")),
        lambda: w.set_joint_damping(j, True, 3, 1.0, 0.0),
        lambda: w.set_joint_damping(9, True, 0, 1.0, 0.0),
    ]
    for k, call in enumerate(calls):
        try:
            call()
        except rp.RPhysError:
            pass
        else:
            raise AssertionError(f"call {k} accepted")
    w.set_joint_axis(j, False, 1, False, 0.0)
    w.set_joint_drive(j, True, 0, 0.5, max_impulse=10.0, velocity=True)
    w.set_joint_drive(j, True, 0)  # cleared
    w.set_joint_damping(j, True, 1, 2.0, 0.5)
    w.step(1.0 / 60.0)
    w.close()


# ---- distance joints
def case_compliant_distance_joint_holds_its_static_stretch(lib):
    """compliant_joint_test.rs:77-112: a 2 kg weight on a compliant distance joint (0.0005 m/N),
    started at its static stretch c m g, stays within 3% of it for 10 s at 60 Hz / 20 iterations,
    240 Hz / 20 and 240 Hz / 4."""
    c, m = 0.0005, 2.0
    stretch = c * m * G
    for hz, iters in ((60.0, 20), (240.0, 20), (240.0, 4)):
        w = _world(lib, 4)
        w.set_iterations(iters, iters)
        p = _body(w, (0.0, 10.0, 0.0), PIN, 1.0, dynamic=False)
        bob = _body(w, (0.0, 9.0 - stretch, 0.0), (0.05, 0.05, 0.05), m / 0.001, sleep=False)
        w.add_distance_joints([(p, bob, (0, 0, 0), (0, 0, 0), 1.0, c, 0.0)])
        worst = 0.0
        for _ in range(int(10.0 * hz)):
            w.step(1.0 / hz)
            s = (10.0 - w.pose(bob)[0][1]) - 1.0
            worst = max(worst, abs(s - stretch) / stretch)
        assert worst < 0.03, f"{hz} Hz, {iters} iterations: stretch departed {100 * worst:.2f}%"
        w.close()


def case_rigid_distance_joint_stays_rigid(lib):
    """compliant_joint_test.rs:114-131: compliance 0 holds a 1 m rod within 2 mm for 10 s."""
    w = _world(lib, 4)
    p = _body(w, (0.0, 10.0, 0.0), PIN, 1.0, dynamic=False)
    bob = _body(w, (1.0, 10.0, 0.0), (0.05, 0.05, 0.05), 1000.0)
    w.add_distance_joints([(p, bob, (0, 0, 0), (0, 0, 0), 1.0, 0.0, 0.0)])
    worst = 0.0
    for _ in range(600):
        w.step(1.0 / 60.0)
        worst = max(worst, abs(float(np.linalg.norm(np.array(w.pose(bob)[0]) - np.array([0.0, 10.0, 0.0]))) - 1.0))
    assert worst < 0.002, f"rigid distance joint stretched {worst:.4f} m"
    w.close()


def _f32(x):
    return np.float32(x)


def _glam_qmul(a, b):
    """glam's SSE2 Quat product (lane order (w0 b + x0 b1) + (y0 b2 + z0 b3)) in f32."""
    ax, ay, az, aw = (_f32(v) for v in a)
    bx, by, bz, bw = (_f32(v) for v in b)
    return ((aw * bx + ax * bw) + (ay * bz - az * by),
            (aw * by - ax * bz) + (ay * bw + az * bx),
            (aw * bz + ax * by) + (-(ay * bx) + az * bw),
            (aw * bw - ax * bx) + (-(ay * by) - az * bz))


DISTANCE_GOLDEN = {  # distance_bits_test.rs:52-55, recorded from the reference binary
    (0, 60.0): 0x87F81A83F9615530, (0, 240.0): 0xE7411745726C1915,
    (1, 60.0): 0x6F111D612DA3E10F, (1, 240.0): 0xED532E5E87913E18,
}


def distance_golden_scene(lib, kind, hz):
    """distance_bits_test.rs:21-48 through the C ABI: a 0.2 x 0.1 x 0.16 m box of density 500 on a
    distance joint from a static pivot at (0, 5, 0) (a 2 cm box here: the FFI gives every body a
    collider; a jointed pair makes no contact), kind 0 rigid at its start length, kind 1 a spring
    (2e-3 m/N) at 0.8 of it; 3 s at hz. Returns bits(): the FNV-1a fold of the box's pose and
    velocity bits."""
    w = lib.world(8, 8)
    w.set_gravity((0.0, -9.81, 0.0))
    w.set_iterations(20, 20)
    p = _body(w, (0.0, 5.0, 0.0), PIN, 1.0, dynamic=False)
    h = _f32(0.3) * _f32(0.5), _f32(0.2) * _f32(0.5)
    qy = (0.0, _f32(math.sin(float(h[0]))), 0.0, _f32(math.cos(float(h[0]))))
    qx = (_f32(math.sin(float(h[1]))), 0.0, 0.0, _f32(math.cos(float(h[1]))))
    rot = tuple(float(v) for v in _glam_qmul(qy, qx))
    start = (0.7, 4.3, 0.2)
    b = _body(w, start, (0.1, 0.05, 0.08), 500.0, rot=rot, lin=(0.0, 0.5, 1.5), ang=(0.4, -1.0, 2.0), sleep=False)
    d = np.array(start, dtype=np.float32) - np.array([0.0, 5.0, 0.0], dtype=np.float32)
    rest = np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
    if kind == 0:
        w.add_distance_joints([(p, b, (0, 0, 0), (0, 0, 0), float(rest), 0.0, 0.0)])
    else:
        w.add_distance_joints([(p, b, (0, 0, 0), (0, 0, 0), float(rest * _f32(0.8)), 2.0e-3, 0.0)])
    dt = float(_f32(1.0) / _f32(hz))
    for _ in range(int(3.0 * hz)):
        w.step(dt)
    (pos, q), (lin, ang) = w.pose(b), w.velocity(b)
    hsh = 0xCBF29CE484222325
    for x in list(pos) + list(q) + list(lin) + list(ang):
        hsh = ((hsh ^ int(np.float32(x).view(np.uint32))) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    w.close()
    return hsh


def case_distance_joint_scenes_keep_the_reference_bits(lib):
    """distance_bits_test.rs:48-63: the reference binary's golden bits, through the C ABI."""
    for (kind, hz), want in sorted(DISTANCE_GOLDEN.items()):
        got = distance_golden_scene(lib, kind, hz)
        assert got == want, f"kind {kind} {hz} Hz: {got:016x}, reference {want:016x}"


def case_distance_joint_api_errors(lib):
    """Argument checks of rphys_ext_add_distance_joints (all-or-nothing)."""
    w = lib.world(4, 4)
    a = _body(w, (0.0, 1.0, 0.0), (0.5, 0.5, 0.5), 1000.0)
    b = _body(w, (2.0, 1.0, 0.0), (0.5, 0.5, 0.5), 1000.0)
    bad = [
        (a, a, (0, 0, 0), (0, 0, 0), 1.0, 0.0, 0.0),
        (a, 99, (0, 0, 0), (0, 0, 0), 1.0, 0.0, 0.0),
        (a, b, (float("nan"), 0, 0), (0, 0, 0), 1.0, 0.0, 0.0),
        (a, b, (0, 0, 0), (0, 0, 0), float("inf"), 0.0, 0.0),
        (a, b, (0, 0, 0), (0, 0, 0), 1.0, -1.0, 0.0),
        (a, b, (0, 0, 0), (0, 0, 0), 1.0, 0.0, -2.0),
    ]
    for j in bad:
        try:
            w.add_distance_joints([(a, b, (0, 0, 0), (0, 0, 0), 2.0, 0.0, 0.0), j])
        except rp.RPhysError:
            pass
        else:
            raise AssertionError(f"accepted {j}")
    assert w.num_joints() == 0
    assert w.add_distance_joints([(a, b, (0.1, 0, 0), (0, 0, 0), 2.0, 1e-3, 5.0)]) == 0
    w.step(1.0 / 60.0)
    w.close()
