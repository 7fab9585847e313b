"""riftphys-rust_b200: Python bindings of the RiftPhys C ABI (v1 + extensions).

The product is ``build/librphys_gpu.so`` in this directory: the reference's C ABI
(crates/riftphys-ffi/src/riftphys_c.h) implemented by C++ host code over hand-written sm_100a
CUDA kernels. This module only declares the ctypes signatures of that ABI, mirroring the
reference's FFI one entry point per function, and gives a thin ``World`` wrapper with the same
names, argument meanings and error codes (an ``RPhysError`` carries the code and the
thread-local message, as ``rphys_last_error_message`` does in crates/riftphys-ffi/src/lib.rs).

``load_product()`` loads the CUDA library and raises if it is missing: there is no CPU
fallback on the product path.
"""
import ctypes
import os
from ctypes import (POINTER, Structure, byref, c_char, c_char_p, c_float, c_int,
                    c_uint8, c_uint32, c_uint64, c_void_p)

HERE = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIB = os.path.join(HERE, "build", "librphys_gpu.so")

RPHYS_OK = 0
RPHYS_ERR_NULL = 1
RPHYS_ERR_INVALID_ID = 2
RPHYS_ERR_CAPACITY = 3
RPHYS_ERR_BAD_ARG = 4
RPHYS_ERR_INTERNAL = 0x80000000
RPHYS_TERRAIN_BODY_ID = 0xFFFFFFFF
RPHYS_BODY_STATIC = 0
RPHYS_BODY_DYNAMIC = 1
SHAPE_SPHERE, SHAPE_BOX, SHAPE_CAPSULE = 0, 1, 2


class Vec3(Structure):
    _fields_ = [("x", c_float), ("y", c_float), ("z", c_float)]


class Quat(Structure):
    _fields_ = [("x", c_float), ("y", c_float), ("z", c_float), ("w", c_float)]


class Isometry(Structure):
    _fields_ = [("pos", Vec3), ("rot", Quat)]


class Velocity(Structure):
    _fields_ = [("lin", Vec3), ("ang", Vec3)]


class Material(Structure):
    _fields_ = [("mu_static", c_float), ("mu_dynamic", c_float), ("restitution", c_float)]


class CapsuleBodyDesc(Structure):
    _fields_ = [("pose", Isometry), ("vel", Velocity), ("radius", c_float), ("half_height", c_float),
                ("mass", c_float), ("body_type", c_uint32), ("material", Material), ("user_tag", c_uint32)]


class BoxBodyDesc(Structure):
    _fields_ = [("pose", Isometry), ("vel", Velocity), ("hx", c_float), ("hy", c_float), ("hz", c_float),
                ("mass", c_float), ("body_type", c_uint32), ("material", Material), ("user_tag", c_uint32)]


class SphereBodyDesc(Structure):
    _fields_ = [("pose", Isometry), ("vel", Velocity), ("radius", c_float), ("mass", c_float),
                ("body_type", c_uint32), ("material", Material), ("user_tag", c_uint32)]


class Hash32(Structure):
    _fields_ = [("bytes", c_uint8 * 32)]


class StepParams(Structure):
    _fields_ = [("size_bytes", c_uint32), ("flags", c_uint32), ("substeps", c_uint32),
                ("solver_iters", c_uint32), ("dt", c_float)]


class ContactEvent(Structure):
    _fields_ = [("body_id_a", c_uint32), ("body_id_b", c_uint32), ("position", Vec3), ("normal", Vec3),
                ("impulse", c_float)]


class HeightfieldDesc(Structure):
    _fields_ = [("size_bytes", c_uint32), ("flags", c_uint32), ("width", c_uint32), ("height", c_uint32),
                ("row_stride", c_uint32), ("cell_size_x", c_float), ("cell_size_z", c_float),
                ("height_scale", c_float), ("height_offset", c_float), ("heights", c_void_p)]


class BodyDescEx(Structure):
    _fields_ = [("pose", Isometry), ("vel", Velocity), ("shape", c_uint32), ("dims", c_float * 3),
                ("density", c_float), ("body_type", c_uint32), ("material_id", c_uint32),
                ("sleep_allowed", c_uint32)]


def desc_array(pos, rot, dims, shape, density, body_type, material=0, sleep_allowed=1, lin=None, ang=None):
    """A numpy array laid out as RPhysBodyDescEx[n] (84 bytes each), built column-wise: for scenes
    of millions of bodies, where one ctypes object per body is too slow."""
    import numpy as np
    n = len(pos)
    a = np.zeros((n, 21), dtype=np.float32)
    a[:, 0:3] = pos
    a[:, 3:7] = rot
    if lin is not None:
        a[:, 7:10] = lin
    if ang is not None:
        a[:, 10:13] = ang
    u = a.view(np.uint32)
    u[:, 13] = shape
    a[:, 14:17] = dims
    a[:, 17] = density
    u[:, 18] = body_type
    u[:, 19] = material
    u[:, 20] = sleep_allowed
    assert a.strides[0] == ctypes.sizeof(BodyDescEx)
    return a


class PairProps(Structure):
    _fields_ = [("mu_s", c_float), ("mu_k", c_float), ("restitution", c_float), ("stribeck_v", c_float)]


class JointDesc(Structure):
    _fields_ = [("kind", c_uint32), ("hinge_axis", c_uint32), ("body_a", c_uint32), ("body_b", c_uint32),
                ("frame_a", Isometry), ("frame_b", Isometry)]


JOINT_BALL = 0
JOINT_HINGE = 1
JOINT_D6 = 2


class RayQuery(Structure):
    _fields_ = [("origin", Vec3), ("dir", Vec3), ("max_distance", c_float), ("ignore_body", c_uint32)]


class RayHit(Structure):
    _fields_ = [("hit", c_uint32), ("body_id", c_uint32), ("fraction", c_float), ("point", Vec3), ("normal", Vec3)]


class CapsuleSweepQuery(Structure):
    _fields_ = [("from_", Vec3), ("to", Vec3), ("radius", c_float), ("half_height", c_float), ("ignore_body", c_uint32)]


class CapsuleSweepHit(Structure):
    _fields_ = [("hit", c_uint32), ("body_id", c_uint32), ("fraction", c_float), ("started_overlapping", c_uint32),
                ("point", Vec3), ("normal", Vec3)]


class PlayerDesc(Structure):
    _fields_ = [("start_pose", Isometry), ("radius", c_float), ("height", c_float), ("speed", c_float)]


class DistanceJointDesc(Structure):
    _fields_ = [("body_a", c_uint32), ("body_b", c_uint32), ("anchor_a", Vec3), ("anchor_b", Vec3),
                ("rest", c_float), ("compliance", c_float), ("damping", c_float)]


class JointDrive(Structure):
    _fields_ = [("target", c_float), ("kp", c_float), ("kd", c_float), ("max_impulse", c_float),
                ("vel_mode", c_uint32)]


class JointLimit(Structure):
    _fields_ = [("joint", c_uint32), ("angular", c_uint32), ("axis", c_uint32), ("enabled", c_uint32),
                ("lo", c_float), ("hi", c_float)]


def joint_array(kind, axis, a, b, fa_pos, fa_rot, fb_pos, fb_rot):
    """A numpy array laid out as RPhysJointDesc[n] (72 bytes each), built column-wise."""
    import numpy as np
    n = len(kind)
    x = np.zeros((n, 18), dtype=np.float32)
    u = x.view(np.uint32)
    u[:, 0] = kind
    u[:, 1] = axis
    u[:, 2] = a
    u[:, 3] = b
    x[:, 4:7] = fa_pos
    x[:, 7:11] = fa_rot
    x[:, 11:14] = fb_pos
    x[:, 14:18] = fb_rot
    assert x.strides[0] == ctypes.sizeof(JointDesc)
    return x


def limit_array(joint, angular, axis, lo, hi):
    """A numpy array laid out as RPhysJointLimit[n] (24 bytes each), every limit enabled."""
    import numpy as np
    n = len(joint)
    x = np.zeros((n, 6), dtype=np.float32)
    u = x.view(np.uint32)
    u[:, 0] = joint
    u[:, 1] = angular
    u[:, 2] = axis
    u[:, 3] = 1
    x[:, 4] = lo
    x[:, 5] = hi
    assert x.strides[0] == ctypes.sizeof(JointLimit)
    return x


class StepStats(Structure):
    _fields_ = [(n, c_uint32) for n in ("pairs", "contacts", "islands", "levels", "max_batch", "warm_matched",
                                        "sweeps", "bounce_rows", "warm_entries", "sleeping", "error_flags")] + \
               [("residual", c_float), ("row_sweeps", c_uint32), ("rows_scheduled", c_uint32)] + \
               [(n, c_uint32) for n in ("groups_shared", "groups_global", "max_group_rows", "max_group_bodies",
                                        "islands_capped", "pred_used", "rows_capped")] + \
               [("res_hist", c_uint32 * 6)]


class Tuning(Structure):
    _fields_ = [("group_rows", c_uint32), ("packed_threads", c_uint32), ("island_threads", c_uint32)]


class ContactRecord(Structure):
    _fields_ = [("a_collider", c_uint32), ("b_collider", c_uint32), ("point", Vec3), ("normal", Vec3),
                ("depth", c_float), ("impulse", c_float), ("level", c_uint32), ("pad", c_uint32)]


# (name, restype, argtypes) of every entry point declared in include/riftphys_c.h and include/rphys_ext.h
ABI = [
    ("rphys_get_abi_version", c_uint32, []),
    ("rphys_get_build_id", c_char_p, []),
    ("rphys_last_error_message", c_char_p, []),
    ("rphys_last_error_copy", c_uint32, [c_char_p, c_uint32, POINTER(c_uint32)]),
    ("rphys_world_create", c_void_p, [c_uint32, c_uint32]),
    ("rphys_world_destroy", None, [c_void_p]),
    ("rphys_world_set_epoch", c_uint32, [c_void_p, c_uint64]),
    ("rphys_world_set_rng_seed", c_uint32, [c_void_p, c_uint64]),
    ("rphys_add_capsule_body", c_uint32, [c_void_p, POINTER(CapsuleBodyDesc), POINTER(c_uint32)]),
    ("rphys_add_box_body", c_uint32, [c_void_p, POINTER(BoxBodyDesc), POINTER(c_uint32)]),
    ("rphys_add_sphere_body", c_uint32, [c_void_p, POINTER(SphereBodyDesc), POINTER(c_uint32)]),
    ("rphys_body_remove", c_uint32, [c_void_p, c_uint32]),
    ("rphys_body_get_pose", c_uint32, [c_void_p, c_uint32, POINTER(Isometry)]),
    ("rphys_body_set_pose", c_uint32, [c_void_p, c_uint32, POINTER(Isometry)]),
    ("rphys_body_get_velocity", c_uint32, [c_void_p, c_uint32, POINTER(Velocity)]),
    ("rphys_body_set_velocity", c_uint32, [c_void_p, c_uint32, POINTER(Velocity)]),
    ("rphys_body_apply_impulse", c_uint32, [c_void_p, c_uint32, Vec3]),
    ("rphys_world_step_ex", c_uint32, [c_void_p, POINTER(StepParams)]),
    ("rphys_world_step", c_uint32, [c_void_p, c_float]),
    ("rphys_world_tick_index", c_uint32, [c_void_p, POINTER(c_uint64)]),
    ("rphys_world_num_bodies", c_uint32, [c_void_p, POINTER(c_uint32)]),
    ("rphys_world_get_step_hash", c_uint32, [c_void_p, POINTER(Hash32)]),
    ("rphys_world_step_and_hash", c_uint32, [c_void_p, c_float, POINTER(Hash32)]),
    ("rphys_world_set_heightfield_i16", c_uint32, [c_void_p, POINTER(HeightfieldDesc), c_float, c_float, c_float]),
    ("rphys_world_set_heightfield_raw32_square", c_uint32,
     [c_void_p, c_void_p, c_uint32, c_float, c_float, c_float, c_float, c_float]),
    ("rphys_world_clear_heightfield", c_uint32, [c_void_p]),
    ("rphys_world_get_contacts", c_uint32, [c_void_p, POINTER(ContactEvent), c_uint32, POINTER(c_uint32)]),
    ("rphys_world_snapshot_create", c_void_p, [c_void_p]),
    ("rphys_world_snapshot_restore", c_uint32, [c_void_p, c_void_p]),
    ("rphys_world_snapshot_free", None, [c_void_p]),
    ("rphys_ext_add_bodies", c_uint32, [c_void_p, POINTER(BodyDescEx), c_uint32, POINTER(c_uint32)]),
    ("rphys_ext_snapshot_restore_exact", c_uint32, [c_void_p, c_void_p]),
    ("rphys_ext_set_warm_model", c_uint32, [c_void_p, c_void_p]),
    ("rphys_ext_set_warm_policy", c_uint32, [c_void_p, c_uint32]),
    ("rphys_ext_set_feature_logging", c_uint32, [c_void_p, c_uint32]),
    ("rphys_ext_get_row_features", c_uint32, [c_void_p, c_void_p, c_void_p, c_uint32, POINTER(c_uint32)]),
    ("rphys_ext_get_row_predictions", c_uint32, [c_void_p, c_void_p, c_uint32, POINTER(c_uint32)]),
    ("rphys_ext_model_create", c_void_p, [c_uint64]),
    ("rphys_ext_model_destroy", None, [c_void_p]),
    ("rphys_ext_model_num_params", c_uint32, []),
    ("rphys_ext_model_get_weights", c_uint32, [c_void_p, c_void_p, c_uint32]),
    ("rphys_ext_model_set_weights", c_uint32, [c_void_p, c_void_p, c_uint32]),
    ("rphys_ext_model_predict", c_uint32, [c_void_p, c_void_p, c_uint32, c_void_p]),
    ("rphys_ext_model_predict_device", c_uint32, [c_void_p, c_void_p, c_uint32, c_void_p, c_uint64]),
    ("rphys_ext_model_gradients", c_uint32, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, POINTER(c_float)]),
    ("rphys_ext_model_train", c_uint32, [c_void_p, c_void_p, c_void_p, c_uint32, c_uint32, c_uint32, c_float,
                                         POINTER(c_float)]),
    ("rphys_ext_batch_add_world", c_uint32, [c_void_p, c_void_p, c_uint32, POINTER(c_uint32), POINTER(c_uint32)]),
    ("rphys_ext_batch_num_worlds", c_uint32, [c_void_p, POINTER(c_uint32)]),
    ("rphys_ext_batch_world_range", c_uint32, [c_void_p, c_uint32, POINTER(c_uint32), POINTER(c_uint32)]),
    ("rphys_ext_batch_get_hashes", c_uint32, [c_void_p, c_uint32, c_uint32, c_void_p]),
    ("rphys_ext_set_pair_props", c_uint32, [c_void_p, c_uint32, c_uint32, POINTER(PairProps)]),
    ("rphys_ext_set_solver_iterations", c_uint32, [c_void_p, c_uint32, c_uint32]),
    ("rphys_ext_set_gravity", c_uint32, [c_void_p, Vec3]),
    ("rphys_ext_set_heightfield_f32", c_uint32,
     [c_void_p, c_uint32, c_uint32, c_float, c_float, c_float, c_float, c_void_p, c_uint32]),
    ("rphys_ext_set_residual_mode", c_uint32, [c_void_p, c_float, c_uint32]),
    ("rphys_ext_step_n", c_uint32, [c_void_p, c_float, c_uint32]),
    ("rphys_ext_get_stats", c_uint32, [c_void_p, POINTER(StepStats)]),
    ("rphys_ext_get_pairs", c_uint32, [c_void_p, c_void_p, c_uint32, POINTER(c_uint32)]),
    ("rphys_ext_get_contact_records", c_uint32, [c_void_p, POINTER(ContactRecord), c_uint32, POINTER(c_uint32)]),
    ("rphys_ext_get_body_states", c_uint32, [c_void_p, c_uint32, c_uint32, c_void_p]),
    ("rphys_ext_profile_enable", c_uint32, [c_void_p, c_uint32]),
    ("rphys_ext_profile_read", c_uint32, [c_void_p, c_void_p, c_void_p, c_uint32, POINTER(c_uint32)]),
    ("rphys_ext_profile_stage_name", c_char_p, [c_uint32]),
    ("rphys_ext_stream_handle", c_uint32, [c_void_p, POINTER(c_uint64)]),
    ("rphys_ext_launch_count", c_uint32, [POINTER(c_uint64)]),
    ("rphys_ext_world_step_hash_noalloc", c_uint32, [c_void_p, POINTER(Hash32)]),
    ("rphys_ext_add_joints", c_uint32, [c_void_p, POINTER(JointDesc), c_uint32, POINTER(c_uint32)]),
    ("rphys_ext_set_joint_limit", c_uint32, [c_void_p, c_uint32, c_uint32, c_uint32, c_uint32, c_float, c_float]),
    ("rphys_ext_num_joints", c_uint32, [c_void_p, POINTER(c_uint32)]),
    ("rphys_ext_set_joint_limits", c_uint32, [c_void_p, c_void_p, c_uint32]),
    ("rphys_world_capsule_sweep", c_uint32, [c_void_p, POINTER(CapsuleSweepQuery), POINTER(CapsuleSweepHit)]),
    ("rphys_world_raycast", c_uint32, [c_void_p, POINTER(RayQuery), POINTER(RayHit)]),
    ("rphys_add_player", c_uint32, [c_void_p, POINTER(PlayerDesc), POINTER(c_uint32)]),
    ("rphys_player_set_input", c_uint32, [c_void_p, c_uint32, Vec3]),
    ("rphys_player_get_pose", c_uint32, [c_void_p, c_uint32, POINTER(Isometry), POINTER(c_uint32)]),
    ("rphys_ext_raycast_batch", c_uint32, [c_void_p, POINTER(RayQuery), c_uint32, POINTER(RayHit)]),
    ("rphys_ext_raycast_exact_batch", c_uint32, [c_void_p, POINTER(RayQuery), c_uint32, POINTER(RayHit)]),
    ("rphys_ext_pack_snapshot", c_uint32, [c_void_p, c_uint64, c_uint64, c_void_p, c_uint64, POINTER(c_uint64),
                                           POINTER(c_uint32)]),
    ("rphys_ext_add_distance_joints", c_uint32, [c_void_p, POINTER(DistanceJointDesc), c_uint32, POINTER(c_uint32)]),
    ("rphys_ext_set_joint_axis", c_uint32, [c_void_p, c_uint32, c_uint32, c_uint32, c_uint32, c_float]),
    ("rphys_ext_set_joint_drive", c_uint32, [c_void_p, c_uint32, c_uint32, c_uint32, POINTER(JointDrive)]),
    ("rphys_ext_set_joint_damping", c_uint32, [c_void_p, c_uint32, c_uint32, c_uint32, c_float, c_float]),
    ("rphys_ext_state_export", c_uint32, [c_void_p, c_void_p, c_uint64, POINTER(c_uint64)]),
    ("rphys_ext_state_import", c_uint32, [c_void_p, c_void_p, c_uint64]),
    ("rphys_ext_set_solve_order", c_uint32, [c_void_p, c_uint32]),
    ("rphys_ext_set_tuning", c_uint32, [c_void_p, POINTER(Tuning)]),
    ("rphys_ext_get_tuning", c_uint32, [c_void_p, POINTER(Tuning)]),
]


class RPhysError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rphys error {code:#x}: {msg}")
        self.code = code
        self.msg = msg


class Lib:
    """A loaded library exporting the RiftPhys C ABI (the CUDA product, or a test oracle)."""

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(f"RiftPhys library not built: {path}")
        self.path = path
        self.dll = ctypes.CDLL(path)
        for name, res, args in ABI:
            f = getattr(self.dll, name)
            f.restype = res
            f.argtypes = args
        self.extra = {}

    def call(self, name, *args):
        r = getattr(self.dll, name)(*args)
        if r != RPHYS_OK:
            msg = self.dll.rphys_last_error_message()
            raise RPhysError(r, msg.decode() if msg else "")
        return r

    def launch_count(self):
        n = c_uint64(0)
        self.call("rphys_ext_launch_count", byref(n))
        return n.value

    def world(self, max_bodies=1024, max_colliders=2048):
        return World(self, max_bodies, max_colliders)

    def model(self, seed=1):
        return WarmModel(self, seed)


def load_product():
    """The CUDA library. Raises if it was not built: the product has no CPU fallback."""
    return Lib(PRODUCT_LIB)


def iso(x=0.0, y=0.0, z=0.0, q=(0.0, 0.0, 0.0, 1.0)):
    return Isometry(Vec3(x, y, z), Quat(*q))


def vel(lin=(0.0, 0.0, 0.0), ang=(0.0, 0.0, 0.0)):
    return Velocity(Vec3(*lin), Vec3(*ang))


class World:
    """Owns one RPhysWorld handle of a Lib."""

    def __init__(self, lib, max_bodies=1024, max_colliders=2048):
        self.lib = lib
        self.h = lib.dll.rphys_world_create(max_bodies, max_colliders)
        if not self.h:
            msg = lib.dll.rphys_last_error_message()
            raise RPhysError(RPHYS_ERR_INTERNAL, msg.decode() if msg else "create failed")

    def close(self):
        if self.h:
            self.lib.dll.rphys_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def c(self, name, *args):
        return self.lib.call(name, self.h, *args)

    # ---- v1
    def add_box(self, pos, he, dynamic=True, mass=1.0, q=(0, 0, 0, 1), v=(0, 0, 0), w=(0, 0, 0)):
        d = BoxBodyDesc(iso(*pos, q=q), vel(v, w), he[0], he[1], he[2], mass,
                        RPHYS_BODY_DYNAMIC if dynamic else RPHYS_BODY_STATIC, Material(0.9, 0.7, 0.0), 0)
        out = c_uint32(0)
        self.c("rphys_add_box_body", byref(d), byref(out))
        return out.value

    def add_sphere(self, pos, r, dynamic=True, mass=1.0, v=(0, 0, 0)):
        d = SphereBodyDesc(iso(*pos), vel(v), r, mass, RPHYS_BODY_DYNAMIC if dynamic else RPHYS_BODY_STATIC,
                           Material(0.9, 0.7, 0.0), 0)
        out = c_uint32(0)
        self.c("rphys_add_sphere_body", byref(d), byref(out))
        return out.value

    def add_capsule(self, pos, r, hh, dynamic=True, mass=1.0, q=(0, 0, 0, 1)):
        d = CapsuleBodyDesc(iso(*pos, q=q), vel(), r, hh, mass, RPHYS_BODY_DYNAMIC if dynamic else RPHYS_BODY_STATIC,
                            Material(0.9, 0.7, 0.0), 0)
        out = c_uint32(0)
        self.c("rphys_add_capsule_body", byref(d), byref(out))
        return out.value

    def step(self, dt, substeps=1):
        p = StepParams(ctypes.sizeof(StepParams), 0, substeps, 0, dt)
        self.c("rphys_world_step_ex", byref(p))

    def step_hash(self, dt):
        h = Hash32()
        self.c("rphys_world_step_and_hash", c_float(dt), byref(h))
        return bytes(h.bytes)

    def hash(self):
        h = Hash32()
        self.c("rphys_world_get_step_hash", byref(h))
        return bytes(h.bytes)

    def hash_noalloc(self):
        """The tick hash through the allocation-free entry point (same digest as hash())."""
        h = Hash32()
        self.c("rphys_ext_world_step_hash_noalloc", byref(h))
        return bytes(h.bytes)

    def pose(self, bid):
        p = Isometry()
        self.c("rphys_body_get_pose", bid, byref(p))
        return (p.pos.x, p.pos.y, p.pos.z), (p.rot.x, p.rot.y, p.rot.z, p.rot.w)

    def velocity(self, bid):
        v = Velocity()
        self.c("rphys_body_get_velocity", bid, byref(v))
        return (v.lin.x, v.lin.y, v.lin.z), (v.ang.x, v.ang.y, v.ang.z)

    def tick(self):
        t = c_uint64(0)
        self.c("rphys_world_tick_index", byref(t))
        return t.value

    def num_bodies(self):
        n = c_uint32(0)
        self.c("rphys_world_num_bodies", byref(n))
        return n.value

    def snapshot(self):
        s = self.lib.dll.rphys_world_snapshot_create(self.h)
        if not s:
            raise RPhysError(RPHYS_ERR_INTERNAL, "snapshot_create failed")
        return s

    def restore(self, snap):
        self.c("rphys_world_snapshot_restore", c_void_p(snap))

    def restore_exact(self, snap):
        self.c("rphys_ext_snapshot_restore_exact", c_void_p(snap))

    def state_export(self):
        """rphys_ext_state_export: the world's dynamic state as bytes (loads into a world of either
        library built with the same bodies, joints and settings)."""
        n = c_uint64(0)
        self.c("rphys_ext_state_export", None, 0, byref(n))
        buf = ctypes.create_string_buffer(max(1, n.value))
        self.c("rphys_ext_state_export", buf, n.value, byref(n))
        return buf.raw[: n.value]

    def state_import(self, blob):
        buf = ctypes.create_string_buffer(blob, len(blob))
        self.c("rphys_ext_state_import", buf, len(blob))

    def free_snapshot(self, snap):
        self.lib.dll.rphys_world_snapshot_free(c_void_p(snap))

    def remove_body(self, bid):
        self.c("rphys_body_remove", bid)

    def apply_impulse(self, bid, j):
        self.c("rphys_body_apply_impulse", bid, Vec3(*j))

    def contacts(self):
        n = c_uint32(0)
        self.c("rphys_world_get_contacts", None, 0, byref(n))
        buf = (ContactEvent * max(1, n.value))()
        self.c("rphys_world_get_contacts", buf, n.value, byref(n))
        return list(buf)[: n.value]

    # ---- extensions
    def add_bodies(self, descs):
        arr = (BodyDescEx * len(descs))(*descs)
        out = c_uint32(0)
        self.c("rphys_ext_add_bodies", arr, len(descs), byref(out))
        return out.value

    def add_bodies_array(self, desc):
        """add_bodies from a desc_array; returns the first body id."""
        out = c_uint32(0)
        self.c("rphys_ext_add_bodies", ctypes.cast(c_void_p(desc.ctypes.data), POINTER(BodyDescEx)), len(desc), byref(out))
        return out.value

    def set_warm_model(self, model):
        """Learned warm start on (a WarmModel) or off (None); the model must outlive its use."""
        self.c("rphys_ext_set_warm_model", c_void_p(model.h) if model is not None else None)
        self._model = model

    def set_warm_policy(self, cold_only):
        self.c("rphys_ext_set_warm_policy", 1 if cold_only else 0)

    def set_feature_logging(self, on):
        self.c("rphys_ext_set_feature_logging", 1 if on else 0)

    def row_features(self):
        import numpy as np
        n = c_uint32(0)
        self.c("rphys_ext_get_row_features", None, None, 0, byref(n))
        f = np.zeros((n.value, 24), np.float32)
        t = np.zeros((n.value, 3), np.float32)
        if n.value:
            self.c("rphys_ext_get_row_features", f.ctypes.data_as(c_void_p), t.ctypes.data_as(c_void_p), n.value, byref(n))
        return f, t

    def row_predictions(self):
        import numpy as np
        n = c_uint32(0)
        self.c("rphys_ext_get_row_predictions", None, 0, byref(n))
        p = np.zeros((n.value, 4), np.float32)
        if n.value:
            self.c("rphys_ext_get_row_predictions", p.ctypes.data_as(c_void_p), n.value, byref(n))
        return p

    def oracle_set_predictions(self, pred4):
        """CPU restatement only: offer these per-contact predictions to the next tick's warm start."""
        import numpy as np
        p = np.ascontiguousarray(pred4, dtype=np.float32)
        f = self.lib.dll.rphys_oracle_set_predictions
        f.argtypes = [c_void_p, c_void_p, c_uint32]
        f.restype = c_uint32
        r = f(self.h, p.ctypes.data_as(c_void_p), len(p))
        if r:
            raise RPhysError(r, "rphys_oracle_set_predictions failed")

    def add_world(self, desc):
        """Appends one world of a batch (desc: a desc_array or a list of BodyDescEx); returns
        (world index, first body id)."""
        if isinstance(desc, list):
            desc = (BodyDescEx * len(desc))(*desc)
            n, ptr = len(desc), ctypes.cast(desc, c_void_p)
        else:
            n, ptr = len(desc), c_void_p(desc.ctypes.data)
        wi, first = c_uint32(0), c_uint32(0)
        self.c("rphys_ext_batch_add_world", ptr, n, byref(wi), byref(first))
        return wi.value, first.value

    def num_worlds(self):
        n = c_uint32(0)
        self.c("rphys_ext_batch_num_worlds", byref(n))
        return n.value

    def world_range(self, k):
        f, n = c_uint32(0), c_uint32(0)
        self.c("rphys_ext_batch_world_range", k, byref(f), byref(n))
        return f.value, n.value

    def world_hashes(self, first=0, count=None):
        count = self.num_worlds() - first if count is None else count
        out = (Hash32 * count)()
        self.c("rphys_ext_batch_get_hashes", first, count, ctypes.cast(out, c_void_p))
        return [bytes(h.bytes) for h in out]

    def add_joints(self, joints):
        """joints: iterable of (kind, body_a, body_b, frame_a, frame_b, hinge_axis) with frames as
        ((x, y, z), (qx, qy, qz, qw)). Returns the first joint id."""
        joints = list(joints)
        arr = (JointDesc * max(1, len(joints)))()
        for i, (kind, a, b, fa, fb, axis) in enumerate(joints):
            arr[i].kind = kind
            arr[i].hinge_axis = axis
            arr[i].body_a = a
            arr[i].body_b = b
            arr[i].frame_a = iso(*fa[0], q=tuple(fa[1]))
            arr[i].frame_b = iso(*fb[0], q=tuple(fb[1]))
        first = c_uint32(0)
        self.c("rphys_ext_add_joints", arr, len(joints), byref(first))
        return first.value

    def raycast(self, origin, d, max_distance, ignore=0):
        """rphys_world_raycast: (hit, body_id, fraction, point, normal)."""
        q = RayQuery(Vec3(*origin), Vec3(*d), max_distance, ignore)
        h = RayHit()
        self.c("rphys_world_raycast", byref(q), byref(h))
        return (bool(h.hit), h.body_id, h.fraction, (h.point.x, h.point.y, h.point.z), (h.normal.x, h.normal.y, h.normal.z))

    def capsule_sweep(self, frm, to, radius, half_height, ignore=0):
        """rphys_world_capsule_sweep: (hit, body_id, fraction, started_overlapping, point, normal)."""
        q = CapsuleSweepQuery(Vec3(*frm), Vec3(*to), radius, half_height, ignore)
        h = CapsuleSweepHit()
        self.c("rphys_world_capsule_sweep", byref(q), byref(h))
        return (bool(h.hit), h.body_id, h.fraction, bool(h.started_overlapping), (h.point.x, h.point.y, h.point.z),
                (h.normal.x, h.normal.y, h.normal.z))

    def add_player(self, pose, radius=0.4, height=1.8, speed=5.0):
        """rphys_add_player: a kinematic capsule controller; returns its 0-based index."""
        d = PlayerDesc(pose, radius, height, speed)
        out = c_uint32(0)
        self.c("rphys_add_player", byref(d), byref(out))
        return out.value

    def player_set_input(self, idx, move_dir):
        self.c("rphys_player_set_input", idx, Vec3(*move_dir))

    def player_pose(self, idx):
        """rphys_player_get_pose: ((x, y, z), (qx, qy, qz, qw), grounded)."""
        p = Isometry()
        g = c_uint32(0)
        self.c("rphys_player_get_pose", idx, byref(p), byref(g))
        return (p.pos.x, p.pos.y, p.pos.z), (p.rot.x, p.rot.y, p.rot.z, p.rot.w), bool(g.value)

    def raycast_batch(self, origins, dirs, max_distance, ignore=None, exact=False):
        """rphys_ext_raycast_batch (or, with exact, rphys_ext_raycast_exact_batch: true shapes) over
        arrays of origins and directions: the hits as a numpy array of 9 float32 columns per ray (hit
        and body id as uint32 bits, fraction, point, normal)."""
        import numpy as np
        n = len(origins)
        q = np.zeros((n, 8), dtype=np.float32)
        q[:, 0:3] = origins
        q[:, 3:6] = dirs
        q[:, 6] = max_distance
        if ignore is not None:
            q[:, 7].view(np.uint32)[:] = ignore
        assert q.strides[0] == ctypes.sizeof(RayQuery)
        out = np.zeros((n, 9), dtype=np.float32)
        assert out.strides[0] == ctypes.sizeof(RayHit)
        self.c("rphys_ext_raycast_exact_batch" if exact else "rphys_ext_raycast_batch",
               ctypes.cast(q.ctypes.data, POINTER(RayQuery)), n,
               ctypes.cast(out.ctypes.data, POINTER(RayHit)))
        return out

    def pack_snapshot(self, tick, epoch):
        """The riftnet wire snapshot of the live bodies: (bytes, chunk count)."""
        n, c = c_uint64(0), c_uint32(0)
        self.c("rphys_ext_pack_snapshot", tick, epoch, None, 0, byref(n), byref(c))
        buf = ctypes.create_string_buffer(max(1, n.value))
        self.c("rphys_ext_pack_snapshot", tick, epoch, buf, n.value, byref(n), byref(c))
        return buf.raw[: n.value], c.value

    def add_distance_joints(self, joints):
        """joints: iterable of (body_a, body_b, anchor_a, anchor_b, rest, compliance, damping), anchors
        (x, y, z) in each body's frame. Returns the first joint id."""
        joints = list(joints)
        arr = (DistanceJointDesc * max(1, len(joints)))()
        for i, (a, b, la, lb, rest, comp, damp) in enumerate(joints):
            arr[i].body_a, arr[i].body_b = a, b
            arr[i].anchor_a, arr[i].anchor_b = Vec3(*la), Vec3(*lb)
            arr[i].rest, arr[i].compliance, arr[i].damping = rest, comp, damp
        first = c_uint32(0)
        self.c("rphys_ext_add_distance_joints", arr, len(joints), byref(first))
        return first.value

    def add_joint_array(self, arr):
        """Adds the joints of a joint_array(). Returns the first joint id."""
        first = c_uint32(0)
        self.c("rphys_ext_add_joints", ctypes.cast(arr.ctypes.data, POINTER(JointDesc)), len(arr), byref(first))
        return first.value

    def set_joint_limit_array(self, arr):
        self.c("rphys_ext_set_joint_limits", arr.ctypes.data_as(c_void_p), len(arr))

    def set_joint_limit(self, joint, angular, axis, lo=None, hi=None):
        on = lo is not None
        self.c("rphys_ext_set_joint_limit", joint, 1 if angular else 0, axis, 1 if on else 0,
               float(lo if on else 0.0), float(hi if on else 0.0))

    def set_joint_axis(self, joint, angular, axis, enabled=True, compliance=0.0):
        self.c("rphys_ext_set_joint_axis", joint, 1 if angular else 0, axis, 1 if enabled else 0, float(compliance))

    def set_joint_drive(self, joint, angular, axis, target=None, kp=0.0, kd=0.0, max_impulse=0.0, velocity=False):
        """A position drive (velocity=False) or a velocity motor on one axis; target=None clears it."""
        d = None if target is None else byref(JointDrive(target, kp, kd, max_impulse, 1 if velocity else 0))
        self.c("rphys_ext_set_joint_drive", joint, 1 if angular else 0, axis, d)

    def set_joint_damping(self, joint, angular, axis, damping=0.0, friction=0.0):
        self.c("rphys_ext_set_joint_damping", joint, 1 if angular else 0, axis, float(damping), float(friction))

    def num_joints(self):
        n = c_uint32(0)
        self.c("rphys_ext_num_joints", byref(n))
        return n.value

    def set_pair_props(self, a, b, mu_s, mu_k, restitution, stribeck_v):
        p = PairProps(mu_s, mu_k, restitution, stribeck_v)
        self.c("rphys_ext_set_pair_props", a, b, byref(p))

    def set_iterations(self, v, p):
        self.c("rphys_ext_set_solver_iterations", v, p)

    def set_gravity(self, g):
        self.c("rphys_ext_set_gravity", Vec3(*g))

    def set_heightfield(self, heights, nx, nz, cell_x, cell_z, origin_x, origin_z, material=4):
        import numpy as np
        h = np.ascontiguousarray(heights, dtype=np.float32)
        assert h.size == nx * nz
        self.c("rphys_ext_set_heightfield_f32", nx, nz, c_float(cell_x), c_float(cell_z), c_float(origin_x),
               c_float(origin_z), h.ctypes.data_as(c_void_p), material)

    def set_tuning(self, group_rows, packed_threads, island_threads):
        """rphys_ext_set_tuning: the velocity solve's launch shapes (no result bit changes)."""
        self.c("rphys_ext_set_tuning", byref(Tuning(group_rows, packed_threads, island_threads)))

    def tuning(self):
        t = Tuning()
        self.c("rphys_ext_get_tuning", byref(t))
        return {"group_rows": t.group_rows, "packed_threads": t.packed_threads, "island_threads": t.island_threads}

    def set_coloured(self, on=True):
        """rphys_ext_set_solve_order: coloured order (on) or the reference's serial order."""
        self.c("rphys_ext_set_solve_order", 1 if on else 0)

    def set_residual_mode(self, tol, max_sweeps):
        self.c("rphys_ext_set_residual_mode", c_float(tol), max_sweeps)

    def step_n(self, dt, n):
        self.c("rphys_ext_step_n", c_float(dt), n)

    def stats(self):
        s = StepStats()
        self.c("rphys_ext_get_stats", byref(s))
        out = {f: getattr(s, f) for f, _ in StepStats._fields_}
        out["res_hist"] = list(out["res_hist"])
        return out

    def pairs(self):
        import numpy as np
        n = c_uint32(0)
        self.c("rphys_ext_get_pairs", None, 0, byref(n))
        buf = np.zeros((max(1, n.value), 2), dtype=np.uint32)
        self.c("rphys_ext_get_pairs", buf.ctypes.data_as(c_void_p), n.value, byref(n))
        return buf[: n.value]

    def contact_records(self):
        n = c_uint32(0)
        self.c("rphys_ext_get_contact_records", None, 0, byref(n))
        buf = (ContactRecord * max(1, n.value))()
        self.c("rphys_ext_get_contact_records", buf, n.value, byref(n))
        return list(buf)[: n.value]

    def stream_handle(self):
        s = c_uint64(0)
        self.c("rphys_ext_stream_handle", byref(s))
        return s.value

    def profile(self, on=True):
        self.c("rphys_ext_profile_enable", 1 if on else 0)

    def profile_read(self):
        """{stage: (total ms, ticks)} since profiling was enabled (CUDA library only)."""
        import numpy as np
        ms = np.zeros(64, dtype=np.float64)
        ticks = np.zeros(64, dtype=np.uint64)
        n = c_uint32(0)
        self.c("rphys_ext_profile_read", ms.ctypes.data_as(c_void_p), ticks.ctypes.data_as(c_void_p), 64, byref(n))
        names = [self.lib.dll.rphys_ext_profile_stage_name(i).decode() for i in range(n.value)]
        return {names[i]: (float(ms[i]), int(ticks[i])) for i in range(n.value)}

    def body_states(self, first=0, count=None):
        import numpy as np
        if count is None:
            count = self.num_bodies() - first
        out = np.zeros((count, 13), dtype=np.float32)
        if count:
            self.c("rphys_ext_get_body_states", first, count, out.ctypes.data_as(c_void_p))
        return out


class WarmModel:
    """The learned warm start's MLP (24 -> 128 -> 128 -> 128 -> 3) on the tensor cores."""

    def __init__(self, lib, seed=1):
        self.lib = lib
        self.h = lib.dll.rphys_ext_model_create(seed)
        if not self.h:
            msg = lib.dll.rphys_last_error_message()
            raise RPhysError(RPHYS_ERR_INTERNAL, msg.decode() if msg else "model create failed")
        self.n_params = lib.dll.rphys_ext_model_num_params()

    def close(self):
        if self.h:
            self.lib.dll.rphys_ext_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weights(self):
        import numpy as np
        w = np.zeros(self.n_params, dtype=np.float32)
        self.lib.call("rphys_ext_model_get_weights", self.h, w.ctypes.data_as(c_void_p), self.n_params)
        return w

    def set_weights(self, w):
        import numpy as np
        w = np.ascontiguousarray(w, dtype=np.float32)
        self.lib.call("rphys_ext_model_set_weights", self.h, w.ctypes.data_as(c_void_p), self.n_params)

    def predict(self, feats):
        import numpy as np
        f = np.ascontiguousarray(feats, dtype=np.float32)
        out = np.zeros((len(f), 3), dtype=np.float32)
        self.lib.call("rphys_ext_model_predict", self.h, f.ctypes.data_as(c_void_p), len(f), out.ctypes.data_as(c_void_p))
        return out

    def predict_device(self, feats_ptr, rows, out_ptr, stream=0):
        """Device pointers (e.g. torch tensors' data_ptr()); runs on `stream` (a cudaStream_t)."""
        self.lib.call("rphys_ext_model_predict_device", self.h, c_void_p(feats_ptr), rows, c_void_p(out_ptr), stream)

    def gradients(self, feats, targets):
        import numpy as np
        f = np.ascontiguousarray(feats, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = c_float(0)
        self.lib.call("rphys_ext_model_gradients", self.h, f.ctypes.data_as(c_void_p), t.ctypes.data_as(c_void_p), len(f),
                      g.ctypes.data_as(c_void_p), byref(loss))
        return g, loss.value

    def train(self, feats, targets, epochs=1, batch=4096, lr=1e-3):
        import numpy as np
        f = np.ascontiguousarray(feats, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        loss = c_float(0)
        self.lib.call("rphys_ext_model_train", self.h, f.ctypes.data_as(c_void_p), t.ctypes.data_as(c_void_p), len(f),
                      epochs, batch, c_float(lr), byref(loss))
        return loss.value
