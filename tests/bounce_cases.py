"""W6 bounce acceptance cases over any library exporting the C ABI (the CPU oracle in
tests/test_oracle_bounce.py, the CUDA library in tests/test_gpu_bounce.py), restated from the
reference's riftphys-world/tests/restitution_toi_test.rs with its bodies, materials, rates and
tolerances: free bodies bounce at their time of impact inside the step, so a rebound's apex is
e^2 h at 60 Hz as well as at 240 Hz. Materials are the ordinals of the material table (Ice 1,
Rubber 2, Concrete 6, Aluminum 13); a pair's restitution is the larger of the two."""
import math

import numpy as np

from conftest import rp

G = 9.81
ICE, RUBBER, CONCRETE, ALUMINUM = 1, 2, 6, 13
E = {RUBBER: 0.8, ALUMINUM: 0.4}  # pair restitution of a material with itself (and over concrete)
ID = (0.0, 0.0, 0.0, 1.0)


def _f32(x):
    return float(np.float32(x))


def _world(lib, gravity=True):
    w = lib.world(16, 16)
    w.set_gravity((0.0, -G if gravity else 0.0, 0.0))
    return w


def _floor(w, mat):
    d = rp.desc_array(np.array([[0.0, -0.5, 0.0]]), np.array([ID]), np.array([[50.0, 0.5, 50.0]]), rp.SHAPE_BOX,
                      np.array([1.0]), np.array([0], dtype=np.uint32), material=mat)
    return w.add_bodies_array(d)


def _ball(w, pos, vel, r, mass, mat):
    """restitution_toi_test.rs:27-33: a sphere of mass `mass`, never asleep."""
    density = np.float32(mass) / (np.float32(4.0 / 3.0) * np.float32(math.pi) * np.float32(r) ** 3)
    d = rp.desc_array(np.array([pos]), np.array([ID]), np.array([[r, 0.0, 0.0]]), rp.SHAPE_SPHERE, np.array([density]),
                      np.array([1], dtype=np.uint32), material=mat, sleep_allowed=0, lin=np.array([vel]))
    return w.add_bodies_array(d)


def _box(w, pos, half, mass, mat, rot=ID):
    """restitution_toi_test.rs:35-42: a box of mass `mass`, never asleep."""
    density = np.float32(mass) / (np.float32(8.0) * np.float32(half[0]) * np.float32(half[1]) * np.float32(half[2]))
    d = rp.desc_array(np.array([pos]), np.array([rot]), np.array([half]), rp.SHAPE_BOX, np.array([density]),
                      np.array([1], dtype=np.uint32), material=mat, sleep_allowed=0)
    return w.add_bodies_array(d)


def _apexes(w, b, hz, secs, n, bottom):
    """restitution_toi_test.rs:44-56: apexes of `bottom` after each of the first n bounces."""
    out, rising, apex = [], False, 0.0
    for _ in range(int(secs * hz)):
        w.step(1.0 / hz)
        y, vy = bottom(), w.velocity(b)[0][1]
        if not rising and vy > 0.0:
            rising, apex = True, y
        if rising:
            apex = max(apex, y)
            if vy < 0.0:
                out.append(apex)
                rising = False
                if len(out) == n:
                    break
    return out


def _ball_apexes(lib, h, mat, hz):
    r = 0.1
    w = _world(lib)
    _floor(w, mat)
    b = _ball(w, (0.0, r + h, 0.0), (0.0, 0.0, 0.0), r, 0.1, mat)
    out = _apexes(w, b, hz, 6.0, 2, lambda: w.pose(b)[0][1] - r)
    w.close()
    return out


def case_fidelity_bounce_reaches_e2_h(lib):
    """restitution_toi_test.rs:66-76: a rubber ball (pair e 0.80) from 1 m rebounds to e^2 h (2%)."""
    e = E[RUBBER]
    for hz in (60.0, 240.0):
        got = _ball_apexes(lib, 1.0, RUBBER, hz)[0]
        assert abs(got - e * e) < 0.02 * e * e, f"{hz} Hz: apex {got:.4}, want {e * e:.4}"


def case_drops_and_second_bounces_reach_e2_h_and_e4_h(lib):
    """restitution_toi_test.rs:78-95: rubber and aluminium balls from 0.3, 1 and 3 m: first apex e^2 h
    (2%), second e^4 h (3%) when the first rebound lands faster than 1 m/s."""
    for hz in (60.0, 240.0):
        for mat in (RUBBER, ALUMINUM):
            e = E[mat]
            for h in (0.3, 1.0, 3.0):
                a = _ball_apexes(lib, h, mat, hz)
                w1, w2 = e * e * h, e ** 4 * h
                assert abs(a[0] - w1) < 0.02 * w1, f"{hz} Hz, e {e}, {h} m: apex {a[0]:.4}, want {w1:.4}"
                if math.sqrt(2.0 * G * w1) > 1.3:
                    assert len(a) > 1, f"{hz} Hz, e {e}, {h} m: no second bounce"
                    assert abs(a[1] - w2) < 0.03 * w2, f"{hz} Hz, e {e}, {h} m: second apex {a[1]:.4}, want {w2:.4}"


DRONE_HALF = (0.25, 0.05, 0.25)


def case_a_falling_drone_bounces(lib):
    """restitution_toi_test.rs:108-137: a 1.2 kg aluminium box landing flat on concrete from 2 m
    rebounds to e^2 h (3%) without turning."""
    e, h, hz = E[ALUMINUM], 2.0, 60.0
    w = _world(lib)
    _floor(w, CONCRETE)
    b = _box(w, (0.0, h + DRONE_HALF[1], 0.0), DRONE_HALF, 1.2, ALUMINUM)
    rising, apex, spin = False, 0.0, 0.0
    for _ in range(int(3.0 * hz)):
        w.step(1.0 / hz)
        (lin, ang), y = w.velocity(b), w.pose(b)[0][1] - DRONE_HALF[1]
        if not rising and lin[1] > 0.0:
            rising = True
        if rising:
            spin = max(spin, float(np.linalg.norm(ang)))
            apex = max(apex, y)
            if lin[1] < 0.0:
                break
    w.close()
    assert abs(apex - e * e * h) < 0.03 * e * e * h, f"drone apex {apex:.4}, want {e * e * h:.4}"
    assert spin < 1e-3, f"the flat drone picked up {spin:.2e} rad/s"


def _box_energy(w, b, mass, half):
    (p, q), (lin, ang) = w.pose(b), w.velocity(b)
    x, y, z, s = q
    r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - s * z), 2 * (x * z + s * y)],
                  [2 * (x * y + s * z), 1 - 2 * (x * x + z * z), 2 * (y * z - s * x)],
                  [2 * (x * z - s * y), 2 * (y * z + s * x), 1 - 2 * (x * x + y * y)]])
    hx, hy, hz_ = half
    inertia = np.diag([mass / 3.0 * (hy * hy + hz_ * hz_), mass / 3.0 * (hx * hx + hz_ * hz_), mass / 3.0 * (hx * hx + hy * hy)])
    iw = r @ inertia @ r.T
    a = np.array(ang)
    return 0.5 * mass * float(np.dot(lin, lin)) + 0.5 * float(a @ iw @ a) + mass * G * p[1]


def case_a_bounce_on_a_resting_box_doesnt_lift_it(lib):
    """restitution_toi_test.rs:160-199: an aluminium box dropped 1 m onto another resting on concrete
    rebounds to e^2 h (3%); the lower box moves less than 1 mm; the pair gains no energy."""
    e = E[ALUMINUM]
    half = (0.2, 0.1, 0.2)
    for hz, m_up in ((60.0, 2.0), (240.0, 2.0), (60.0, 0.2), (240.0, 0.2)):
        w = _world(lib)
        _floor(w, CONCRETE)
        low = _box(w, (0.0, 0.1, 0.0), half, 2.0, ALUMINUM)
        up = _box(w, (0.0, 1.3, 0.0), half, m_up, ALUMINUM)
        total = lambda: _box_energy(w, low, 2.0, half) + _box_energy(w, up, m_up, half)
        e0 = total()
        lo, hi, worst = 1e9, -1e9, -1e9
        rising, apex, done = False, 0.0, False
        for _ in range(int(1.5 * hz)):
            w.step(1.0 / hz)
            y = w.pose(low)[0][1]
            lo, hi = min(lo, y), max(hi, y)
            worst = max(worst, total())
            yu, vu = w.pose(up)[0][1] - 0.3, w.velocity(up)[0][1]
            if not done and not rising and vu > 0.0:
                rising = True
            if not done and rising:
                apex = max(apex, yu)
                if vu < 0.0:
                    done = True
        w.close()
        want = e * e
        assert abs(apex - want) < 0.03 * want, f"{hz} Hz, {m_up} kg: rebound {apex:.4}, want {want:.4}"
        assert hi - lo < 1e-3, f"{hz} Hz, {m_up} kg: the lower box moved {hi - lo:.4} m"
        assert worst <= e0 * 1.001 + 1e-4, f"{hz} Hz: energy rose from {e0:.4} to {worst:.4} J"


def case_head_on_in_zero_g_matches_the_closed_form(lib):
    """restitution_toi_test.rs:201-223: two aluminium balls closing at 4 m/s in zero g leave with the
    1-D closed-form velocities (1%) and gap (2 mm)."""
    e = E[ALUMINUM]
    m1, m2, v1, v2, r = 1.0, 2.0, 3.0, -1.0, 0.1
    for hz in (60.0, 240.0):
        w = _world(lib, gravity=False)
        a = _ball(w, (0.0, 1.0, 0.0), (v1, 0.0, 0.0), r, m1, ALUMINUM)
        b = _ball(w, (2.0 * r + 0.83, 1.0, 0.0), (v2, 0.0, 0.0), r, m2, ALUMINUM)
        t_end = 0.5
        for _ in range(int(round(t_end * hz))):
            w.step(1.0 / hz)
        p = m1 * v1 + m2 * v2
        want1 = (p + m2 * e * (v2 - v1)) / (m1 + m2)
        want2 = (p + m1 * e * (v1 - v2)) / (m1 + m2)
        got1, got2 = w.velocity(a)[0][0], w.velocity(b)[0][0]
        gap = w.pose(b)[0][0] - w.pose(a)[0][0] - 2.0 * r
        want_gap = e * (v1 - v2) * (t_end - 0.83 / (v1 - v2))
        w.close()
        assert abs(got1 - want1) < 0.01 * abs(want1), f"{hz} Hz: v1 {got1:.4}, want {want1:.4}"
        assert abs(got2 - want2) < 0.01 * abs(want2), f"{hz} Hz: v2 {got2:.4}, want {want2:.4}"
        assert abs(gap - want_gap) < 2e-3, f"{hz} Hz: gap {gap:.4}, want {want_gap:.4}"


def case_rollback_across_a_bounce_replays(lib):
    """restitution_toi_test.rs:225-241: a tilted box snapshotted just before it lands on concrete
    replays the 30 ticks across its bounce hash for hash."""
    hz = 60.0
    w = _world(lib)
    _floor(w, CONCRETE)
    th = 0.2
    b = _box(w, (0.0, 1.05, 0.0), DRONE_HALF, 1.2, ALUMINUM, rot=(0.0, 0.0, math.sin(th / 2), math.cos(th / 2)))
    for _ in range(24):
        w.step(1.0 / hz)
    snap = w.snapshot()
    first = []
    for _ in range(30):
        w.step(1.0 / hz)
        first.append(w.hash())
    w.restore_exact(snap)
    again = []
    for _ in range(30):
        w.step(1.0 / hz)
        again.append(w.hash())
    w.free_snapshot(snap)
    w.close()
    assert first == again, "replay across a bounce diverged"


def case_a_bounce_on_a_two_box_stack_moves_neither(lib):
    """restitution_toi_test.rs:312-358: an aluminium box dropped 1 m onto a two-box stack on concrete
    rebounds to e^2 h (2%); the stack's boxes move less than 0.1 mm up to the apex."""
    e = E[ALUMINUM]
    half = (0.2, 0.1, 0.2)
    for hz in (60.0, 240.0):
        w = _world(lib)
        _floor(w, CONCRETE)
        c = _box(w, (0.0, 0.1, 0.0), half, 2.0, ALUMINUM)
        b = _box(w, (0.0, 0.3, 0.0), half, 2.0, ALUMINUM)
        a = _box(w, (0.0, 1.5, 0.0), half, 2.0, ALUMINUM)
        rb, rc = [1e9, -1e9], [1e9, -1e9]
        rising, apex, done = False, 0.0, False
        for _ in range(int(1.5 * hz)):
            w.step(1.0 / hz)
            if not done:
                yb, yc = w.pose(b)[0][1], w.pose(c)[0][1]
                rb = [min(rb[0], yb), max(rb[1], yb)]
                rc = [min(rc[0], yc), max(rc[1], yc)]
            ya, va = w.pose(a)[0][1] - 0.5, w.velocity(a)[0][1]
            if not done and not rising and va > 0.0:
                rising = True
            if not done and rising:
                apex = max(apex, ya)
                if va < 0.0:
                    done = True
        w.close()
        assert rb[1] - rb[0] < 1e-4, f"{hz} Hz: B moved {rb[1] - rb[0]:.5} m"
        assert rc[1] - rc[0] < 1e-4, f"{hz} Hz: C moved {rc[1] - rc[0]:.5} m"
        assert abs(apex - e * e) < 0.02 * e * e, f"{hz} Hz: the top box rebounded {apex:.4}, want {e * e:.4}"
