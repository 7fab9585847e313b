"""Seeded synthetic scenes for the benchmark configurations and the parity tests.

All randomness comes from a project-written splitmix64 generator, so the same seed gives the same
f32 inputs on every machine; the scenes are built through the C ABI of whichever library the
``World`` wraps (the CUDA product or the CPU restatement used as a checker).

box_drop      1,000 boxes (half-extent 0.5 m, 1 kg, mu 0.5, e 0) on a 10x10x10 grid at 1.1 m pitch,
              jitter U[-0.05, 0.05] m, yaw U[0, 2 pi), bottom layer 1 m above a static 50x0.5x50 ground
              box, dt 1/60, 8 velocity and 8 position iterations.
batch         independent worlds for one batched launch: body counts log-uniform in [n_min, n_max],
              alternately a square box pyramid (brick half-extent U[0.25, 0.75] m per world) and a
              random pile (half-extents U[0.25, 0.75] m per box, random yaw, dropped from a grid), each
              on its own static 50x0.5x50 ground box; density 1000, dt 1/60, 16 iterations.
ragdolls      humanoids of 15 capsules (radius U[0.05, 0.12] m, segment U[0.2, 0.5] m, mass U[1, 8] kg
              through the density) and 14 joints each: ball joints with swing limits of +-45 degrees
              about joint-frame y and z (two per-axis limits: the reference has no cone limit) and
              hinges about joint-frame z limited to [-120, 0] degrees; dropped with random yaw and a
              random initial velocity onto a 128 x 128 heightfield of the terrain scene's form;
              dt 1/120, 24 velocity and 24 position iterations.
terrain       bodies (40% spheres r U[0.2,0.6], 30% capsules r U[0.15,0.4] hh U[0.3,0.8], 30% boxes
              he U[0.2,0.7], density 1000) at uniform positions in a square of side `area` x [0, 60] m,
              lifted above the terrain, velocities N(0,1) per axis, falling onto a heightfield
              h = 6 sin(x/37) cos(z/53) + 2 valuenoise(x/8, z/8), 1 m spacing; dt 1/60, 20 iterations.
"""
import math

import numpy as np

MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed):
        self.s = seed & MASK64

    def next_u64(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self, lo=0.0, hi=1.0):
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))

    def normal(self):
        u1 = max(self.uniform(), 1e-300)
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def _yaw_quat(theta):
    return (0.0, math.sin(theta * 0.5), 0.0, math.cos(theta * 0.5))


def _rand_quat(rng):
    # uniform random rotation (Shoemake)
    u1, u2, u3 = rng.uniform(), rng.uniform(), rng.uniform()
    a, b = math.sqrt(1 - u1), math.sqrt(u1)
    return (a * math.sin(2 * math.pi * u2), a * math.cos(2 * math.pi * u2),
            b * math.sin(2 * math.pi * u3), b * math.cos(2 * math.pi * u3))


def box_drop(rp, w, n_side=10, pitch=1.1, seed=1, iterations=(8, 8), sleep_allowed=True):
    """Builds the box-drop scene into World ``w``; returns (dt, body count)."""
    rng = SplitMix64(seed)
    w.set_pair_props(0, 0, 0.5, 0.5, 0.0, 0.08)
    w.set_iterations(*iterations)
    descs = [rp.BodyDescEx(rp.iso(0.0, -0.5, 0.0), rp.vel(), rp.SHAPE_BOX, (50.0, 0.5, 50.0), 0.0,
                           rp.RPHYS_BODY_STATIC, 0, 1)]
    off = (n_side - 1) * 0.5
    for iy in range(n_side):
        for iz in range(n_side):
            for ix in range(n_side):
                x = (ix - off) * pitch + rng.uniform(-0.05, 0.05)
                y = 1.0 + 0.5 + iy * pitch + rng.uniform(-0.05, 0.05)
                z = (iz - off) * pitch + rng.uniform(-0.05, 0.05)
                q = _yaw_quat(rng.uniform(0.0, 2.0 * math.pi))
                # MassProps::from_box_density(he, 1 / (8 * 0.125)): 1 kg
                descs.append(rp.BodyDescEx(rp.iso(x, y, z, q=q), rp.vel(), rp.SHAPE_BOX, (0.5, 0.5, 0.5), 1.0,
                                           rp.RPHYS_BODY_DYNAMIC, 0, 1 if sleep_allowed else 0))
    w.add_bodies(descs)
    return 1.0 / 60.0, len(descs)


def value_noise(x, z, seed):
    """Seeded lattice value noise with smoothstep bilinear interpolation (numpy, vectorised)."""
    xi, zi = np.floor(x).astype(np.int64), np.floor(z).astype(np.int64)
    fx, fz = x - xi, z - zi

    def lat(ix, iz):
        with np.errstate(over="ignore"):
            h = (ix.astype(np.uint64) * np.uint64(0x27D4EB2F165667C5)
                 + iz.astype(np.uint64) * np.uint64(0x165667B19E3779F9)
                 + np.uint64((seed * 0x9E3779B97F4A7C15) & MASK64))
            h ^= h >> np.uint64(29)
            h = h * np.uint64(0xBF58476D1CE4E5B9)
            h ^= h >> np.uint64(32)
        return (h >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))

    sx, sz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)
    a, b = lat(xi, zi), lat(xi + 1, zi)
    c, d = lat(xi, zi + 1), lat(xi + 1, zi + 1)
    return (a * (1 - sx) + b * sx) * (1 - sz) + (c * (1 - sx) + d * sx) * sz


def heightfield(n=512, spacing=1.0, seed=7):
    origin = -0.5 * (n - 1) * spacing
    g = origin + spacing * np.arange(n, dtype=np.float64)
    X, Z = np.meshgrid(g, g, indexing="xy")  # row-major, x fastest
    h = 6.0 * np.sin(X / 37.0) * np.cos(Z / 53.0) + 2.0 * value_noise(X / 8.0, Z / 8.0, seed)
    return h.astype(np.float32), origin


def terrain(rp, w, n_bodies=100_000, hf_n=512, area=400.0, seed=2, iterations=(20, 20)):
    """Builds the mixed-shape terrain scene into World ``w``; returns (dt, body count)."""
    rng = SplitMix64(seed)
    h, origin = heightfield(hf_n, 1.0, seed)
    w.set_heightfield(h, hf_n, hf_n, 1.0, 1.0, origin, origin, material=4)  # Grit, as the FFI's terrain
    # restitution 0 on every pair the scene uses; friction from the material table
    w.set_pair_props(0, 0, 0.6, 0.5, 0.0, 0.08)
    w.set_pair_props(0, 4, 0.883176, 0.724569, 0.0, 0.1)
    w.set_iterations(*iterations)
    hmax = float(h.max())
    descs = []
    half = 0.5 * area
    for _ in range(n_bodies):
        kind = rng.uniform()
        if kind < 0.4:
            shape, dims, bound = rp.SHAPE_SPHERE, (rng.uniform(0.2, 0.6), 0.0, 0.0), None
            bound = dims[0]
        elif kind < 0.7:
            r, hh = rng.uniform(0.15, 0.4), rng.uniform(0.3, 0.8)
            shape, dims, bound = rp.SHAPE_CAPSULE, (r, hh, 0.0), r + hh
        else:
            he = (rng.uniform(0.2, 0.7), rng.uniform(0.2, 0.7), rng.uniform(0.2, 0.7))
            shape, dims, bound = rp.SHAPE_BOX, he, math.sqrt(he[0] ** 2 + he[1] ** 2 + he[2] ** 2)
        x, z = rng.uniform(-half, half), rng.uniform(-half, half)
        y = rng.uniform(0.0, 60.0)
        # lift above the local terrain (the heightfield's maximum bounds it from above)
        y = max(y, hmax + bound + 0.1)
        q = _rand_quat(rng)
        v = (rng.normal(), rng.normal(), rng.normal())
        descs.append(rp.BodyDescEx(rp.iso(x, y, z, q=q), rp.vel(v), shape, dims, 1000.0, rp.RPHYS_BODY_DYNAMIC, 0, 1))
    w.add_bodies(descs)
    return 1.0 / 60.0, len(descs)


def batch_world_descs(rp, k, seed=3, n_min=16, n_max=4096):
    """World k of the batched-worlds scene as an RPhysBodyDescEx array (ground box first)."""
    rng = np.random.Generator(np.random.PCG64([seed, k]))
    n = int(math.floor(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
    n = max(n_min, min(n, n_max))
    pos = np.zeros((n + 1, 3)); rot = np.zeros((n + 1, 4)); rot[:, 3] = 1.0
    dims = np.zeros((n + 1, 3)); btype = np.ones(n + 1, dtype=np.uint32); dens = np.full(n + 1, 1000.0)
    pos[0] = (0.0, -0.5, 0.0); dims[0] = (50.0, 0.5, 50.0); btype[0] = 0; dens[0] = 0.0
    if k % 2 == 0:
        # square pyramid, filled bottom-up, bricks of one size per world
        he = rng.uniform(0.25, 0.75)
        b = 1
        while sum(j * j for j in range(1, b + 1)) < n:
            b += 1
        pts = []
        for layer in range(b):
            m = b - layer
            for iz in range(m):
                for ix in range(m):
                    pts.append(((ix - (m - 1) * 0.5) * 2.02 * he, he + layer * (2.0 * he + 0.001),
                                (iz - (m - 1) * 0.5) * 2.02 * he))
        pos[1:] = np.array(pts[:n])
        dims[1:] = he
    else:
        # random pile: a grid of falling boxes, random sizes and yaw
        side = max(2, int(math.ceil(n ** (1.0 / 3.0))))
        idx = np.arange(n)
        ix, iz, iy = idx % side, (idx // side) % side, idx // (side * side)
        pos[1:, 0] = (ix - (side - 1) * 0.5) * 1.6 + rng.uniform(-0.05, 0.05, n)
        pos[1:, 1] = 1.0 + iy * 1.6 + rng.uniform(-0.05, 0.05, n)
        pos[1:, 2] = (iz - (side - 1) * 0.5) * 1.6 + rng.uniform(-0.05, 0.05, n)
        dims[1:] = rng.uniform(0.25, 0.75, (n, 3))
        th = rng.uniform(0.0, 2.0 * math.pi, n)
        rot[1:, 1] = np.sin(th * 0.5); rot[1:, 3] = np.cos(th * 0.5)
    return rp.desc_array(pos, rot, dims, rp.SHAPE_BOX, dens, btype)


def batch_setup(w, iterations=(16, 16)):
    """Shared settings of the batched-worlds scene (also applied to each oracle world)."""
    w.set_pair_props(0, 0, 0.5, 0.5, 0.0, 0.08)
    w.set_iterations(*iterations)
    return 1.0 / 60.0


# ---- ragdolls
# bone: (parent, direction the capsule's local y takes, attach: the parent's end (+1 / -1 along its
# local y), its centre (0), or a shoulder (+2 / -2: beside its top end, clear of the head), joint
# kind (0 ball, 1 hinge) to the parent, hinge axis of the joint frame)
_BONES = [
    (-1, (1, 0, 0), 0, 0, 2),    # 0 pelvis (horizontal)
    (0, (0, 1, 0), 0, 0, 2),     # 1 chest
    (1, (0, 1, 0), 1, 0, 2),     # 2 head
    (1, (-1, 0, 0), 2, 0, 2),    # 3 left upper arm (shoulder beside the top of the chest)
    (3, (-1, 0, 0), 1, 1, 2),    # 4 left forearm (elbow hinge about z)
    (4, (-1, 0, 0), 1, 0, 2),    # 5 left hand
    (1, (1, 0, 0), -2, 0, 2),    # 6 right upper arm
    (6, (1, 0, 0), 1, 1, 2),     # 7 right forearm
    (7, (1, 0, 0), 1, 0, 2),     # 8 right hand
    (0, (0, -1, 0), -1, 0, 2),   # 9 left thigh (hip at the pelvis' -x end)
    (9, (0, -1, 0), 1, 1, 0),    # 10 left shin (knee hinge about x)
    (10, (0, 0, 1), 1, 1, 0),    # 11 left foot (ankle hinge about x)
    (0, (0, -1, 0), 1, 0, 2),    # 12 right thigh (hip at the pelvis' +x end)
    (12, (0, -1, 0), 1, 1, 0),   # 13 right shin
    (13, (0, 0, 1), 1, 1, 0),    # 14 right foot
]
_S45 = math.sqrt(0.5)
_DIR_Q = {(0, 1, 0): (0.0, 0.0, 0.0, 1.0), (0, -1, 0): (0.0, 0.0, 1.0, 0.0),
          (1, 0, 0): (0.0, 0.0, -_S45, _S45), (-1, 0, 0): (0.0, 0.0, _S45, _S45),
          (0, 0, 1): (_S45, 0.0, 0.0, _S45)}


def _qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return (aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
            aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz)


def _qrot(q, v):
    x, y, z, w = q
    u = (x, y, z)
    uv = (u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0])
    uuv = (u[1] * uv[2] - u[2] * uv[1], u[2] * uv[0] - u[0] * uv[2], u[0] * uv[1] - u[1] * uv[0])
    return tuple(v[i] + 2.0 * (w * uv[i] + uuv[i]) for i in range(3))


def _conj(q):
    return (-q[0], -q[1], -q[2], q[3])


def ragdoll_parts(rng, origin, yaw, v0):
    """One humanoid: body rows (pos, rot, (r, hh), density, lin) and joints (kind, axis, parent,
    child, frame a, frame b, limits [(angular, axis, lo, hi)]), indices local to the ragdoll."""
    bodies, joints = [], []
    qy = (0.0, math.sin(0.5 * yaw), 0.0, math.cos(0.5 * yaw))
    ends = []  # per bone: (centre, local rot, half length to the end = hh + r)
    for k, (par, d, attach, kind, hax) in enumerate(_BONES):
        r = rng.uniform(0.05, 0.12)
        hh = 0.5 * rng.uniform(0.2, 0.5)
        m = rng.uniform(1.0, 8.0)
        vol = math.pi * r * r * 2.0 * hh + 4.0 / 3.0 * math.pi * r ** 3
        q = _DIR_Q[d]
        if par < 0:
            c = (0.0, 0.0, 0.0)
        else:
            pc, pq, pe, pr = ends[par]
            if abs(attach) == 2:  # shoulder: below the top end, out to the side by the chest's radius
                la = (-math.copysign(1.0, attach) * (pr + 0.1), pe - pr, 0.0)
            else:
                la = (0.0, attach * pe, 0.0)
            a = tuple(pc[i] + _qrot(pq, la)[i] for i in range(3))
            c = tuple(a[i] + d[i] * (hh + r) for i in range(3))
            fa = (la, _conj(pq))
            fb = ((0.0, -(hh + r), 0.0), _conj(q))
            if kind == 0:
                lim = [(1, 1, -math.pi / 4, math.pi / 4), (1, 2, -math.pi / 4, math.pi / 4)]
            else:
                lim = [(1, hax, -2.0 * math.pi / 3.0, 0.0)]
            joints.append((kind, hax, par, k, fa, fb, lim))
        ends.append((c, q, hh + r, r))
        wc = _qrot(qy, c)
        bodies.append(((origin[0] + wc[0], origin[1] + wc[1], origin[2] + wc[2]), _qmul(qy, q), (r, hh), m / vol, v0))
    return bodies, joints


def ragdoll_arrays(rp, n, seed, area, base_id=1, y0=None, hf=None):
    """n ragdolls as (body desc array, joint desc array, limit array); joint and body ids assume
    the bodies get consecutive ids from base_id and the joints from 0."""
    rng = SplitMix64(seed)
    pos, rot, dims, dens, lin = [], [], [], [], []
    kinds, axes, ja, jb, fap, faq, fbp, fbq = [], [], [], [], [], [], [], []
    lj, la, lx, llo, lhi = [], [], [], [], []
    half = 0.5 * area
    for i in range(n):
        x, z = rng.uniform(-half, half), rng.uniform(-half, half)
        y = (y0 if y0 is not None else 0.0) + rng.uniform(0.5, 3.0)
        if hf is not None:
            y += hf(x, z)
        yaw = rng.uniform(0.0, 2.0 * math.pi)
        v0 = (rng.normal(), rng.normal() - 1.0, rng.normal())
        bodies, joints = ragdoll_parts(rng, (x, y, z), yaw, v0)
        b0 = len(pos)
        for (p, q, (r, hh), de, v) in bodies:
            pos.append(p); rot.append(q); dims.append((r, hh, 0.0)); dens.append(de); lin.append(v)
        for (kind, axis, par, ch, fa, fb, lim) in joints:
            j = len(kinds)
            kinds.append(kind); axes.append(axis)
            ja.append(base_id + b0 + par); jb.append(base_id + b0 + ch)
            fap.append(fa[0]); faq.append(fa[1]); fbp.append(fb[0]); fbq.append(fb[1])
            for (ang, ax, lo, hi) in lim:
                lj.append(j); la.append(ang); lx.append(ax); llo.append(lo); lhi.append(hi)
    nb = len(pos)
    bd = rp.desc_array(np.array(pos), np.array(rot), np.array(dims), rp.SHAPE_CAPSULE, np.array(dens),
                       np.ones(nb, dtype=np.uint32), lin=np.array(lin))
    jd = rp.joint_array(np.array(kinds), np.array(axes), np.array(ja), np.array(jb), np.array(fap), np.array(faq),
                        np.array(fbp), np.array(fbq))
    ld = rp.limit_array(np.array(lj), np.array(la), np.array(lx), np.array(llo), np.array(lhi))
    return bd, jd, ld


def ragdoll_muscles(w, jd, j0):
    """Drives, springs, dampers and friction on the joints of a ragdoll_arrays() joint array added
    from joint id j0: each ball joint's twist a damped spring (compliance 0.05, damping 0.4; XPBD's
    Kelvin-Voigt row) and its swing axes damped (0.3) with friction (0.05); elbows held by a position
    drive at -0.5 rad, knees turned by a velocity motor (0.3 rad/s, at most 0.5 N m s a tick), ankles
    damped with friction."""
    u = jd.view(np.uint32)
    for k in range(len(jd)):
        j, kind, axis = j0 + k, int(u[k, 0]), int(u[k, 1])
        if kind == 0:
            w.set_joint_axis(j, True, 0, True, 0.05)
            w.set_joint_damping(j, True, 0, 0.4, 0.0)
            w.set_joint_damping(j, True, 1, 0.3, 0.05)
            w.set_joint_damping(j, True, 2, 0.3, 0.05)
        elif axis == 2:
            w.set_joint_drive(j, True, 2, -0.5, max_impulse=1000.0)
        elif k % 14 in (9, 12):  # shins (the joint of bone k + 1)
            w.set_joint_drive(j, True, 0, 0.3, max_impulse=0.5, velocity=True)
        else:
            w.set_joint_damping(j, True, 0, 0.2, 0.02)


def ragdolls(rp, w, n_ragdolls=100, hf_n=128, seed=5, iterations=(24, 24), flat_area=None, muscles=False):
    """Builds the ragdoll scene into World ``w``; returns (dt, body count, joint count). With
    flat_area, the ragdolls fall in a square of that side onto a static ground box instead; with
    muscles, ragdoll_muscles() sets drives, springs and dampers on the joints."""
    w.set_pair_props(0, 0, 0.6, 0.5, 0.0, 0.08)
    w.set_pair_props(0, 4, 0.883176, 0.724569, 0.0, 0.1)
    w.set_iterations(*iterations)
    if flat_area is None:
        h, origin = heightfield(hf_n, 1.0, seed)
        w.set_heightfield(h, hf_n, hf_n, 1.0, 1.0, origin, origin, material=4)
        y0, area = float(h.max()) + 1.0, 0.8 * (hf_n - 1)
    else:
        g = rp.desc_array(np.array([[0.0, -0.5, 0.0]]), np.array([[0.0, 0.0, 0.0, 1.0]]), np.array([[50.0, 0.5, 50.0]]),
                          rp.SHAPE_BOX, np.array([0.0]), np.array([0], dtype=np.uint32))
        w.add_bodies_array(g)
        y0, area = 0.5, flat_area
    first = w.num_bodies() + 1
    bd, jd, ld = ragdoll_arrays(rp, n_ragdolls, seed, area, base_id=first, y0=y0)
    w.add_bodies_array(bd)
    j0 = w.add_joint_array(jd)
    if j0:
        ld[:, 0].view(np.uint32)[:] += j0
    w.set_joint_limit_array(ld)
    if muscles:
        ragdoll_muscles(w, jd, j0)
    return 1.0 / 120.0, w.num_bodies(), len(jd)
