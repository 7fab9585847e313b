"""rphys_world_get_contacts (crates/riftphys-ffi/src/lib.rs:1801-1878): the last tick's culled contacts
as RPhysContactEvent (body ids 1-based, 0xFFFFFFFF for the terrain, point, normal, accumulated normal
impulse). Cases run on any library with the C ABI (the CUDA library and the CPU restatement)."""
import ctypes

import numpy as np

from conftest import rp, scenes


def _call(w, buf, cap, count):
    return w.lib.dll.rphys_world_get_contacts(w.h, buf, cap, count)


def case_count_only_with_a_null_buffer(lib):
    w = lib.world(64, 64)
    dt, _ = scenes.box_drop(rp, w, n_side=3)
    n = ctypes.c_uint32(123)
    assert _call(w, None, 0, ctypes.byref(n)) == rp.RPHYS_OK
    assert n.value == 0                                   # nothing stepped yet
    for _ in range(90):
        w.step(dt)
    assert _call(w, None, 0, ctypes.byref(n)) == rp.RPHYS_OK
    assert n.value == w.stats()["contacts"] > 0


def case_null_world_or_count(lib):
    n = ctypes.c_uint32(0)
    assert lib.dll.rphys_world_get_contacts(None, None, 0, ctypes.byref(n)) == rp.RPHYS_ERR_NULL
    w = lib.world(8, 8)
    assert _call(w, None, 0, None) == rp.RPHYS_ERR_NULL


def case_truncates_to_the_buffer_capacity(lib):
    w = lib.world(64, 64)
    dt, _ = scenes.box_drop(rp, w, n_side=3)
    for _ in range(90):
        w.step(dt)
    full = w.contacts()
    buf = (rp.ContactEvent * 8)()
    for e in buf:
        e.body_id_a = 77
    n = ctypes.c_uint32(0)
    assert _call(w, buf, 3, ctypes.byref(n)) == rp.RPHYS_OK
    assert n.value == len(full) > 3                       # the full count, whatever the capacity
    for k in range(3):
        assert bytes(buf[k]) == bytes(full[k])
    assert all(buf[k].body_id_a == 77 for k in range(3, 8))  # nothing written past the capacity


def case_terrain_contacts_carry_the_sentinel(lib):
    w = lib.world(64, 64)
    h = np.zeros((16, 16), dtype=np.float32)
    w.set_heightfield(h, 16, 16, 1.0, 1.0, -8.0, -8.0, material=4)
    w.set_pair_props(0, 4, 0.8, 0.7, 0.0, 0.1)
    w.add_box((0.0, 0.6, 0.0), (0.5, 0.5, 0.5), mass=8.0)
    w.add_sphere((2.0, 0.4, 1.0), 0.4, mass=1.0)
    dt = 1.0 / 60.0
    for _ in range(120):
        w.step(dt)
    ev = w.contacts()
    assert ev and all(e.body_id_b == rp.RPHYS_TERRAIN_BODY_ID for e in ev)
    assert {e.body_id_a for e in ev} == {1, 2}
    for e in ev:   # the box-triangle normal points from the box into the ground, the sphere's out of it
        assert abs(e.normal.y) > 0.99 and abs(e.position.y) < 0.06 and e.impulse >= 0.0
    # resting: the box's normal impulses carry its weight over the tick (1500 kg/m^3 from the FFI)
    box = sum(e.impulse for e in ev if e.body_id_a == 1)
    assert abs(box - 1500.0 * 1.0 * 9.81 * dt) < 0.05 * 1500.0 * 9.81 * dt


def case_pairs_use_one_based_ids_in_contact_order(lib):
    w = lib.world(64, 64)
    dt, _ = scenes.box_drop(rp, w, n_side=3)
    for _ in range(90):
        w.step(dt)
    ev = w.contacts()
    recs = w.contact_records()
    assert len(ev) == len(recs)
    for e, r in zip(ev, recs):
        assert e.body_id_a == r.a_collider + 1                 # one collider per body
        assert e.body_id_b == (r.b_collider + 1 if r.b_collider != 0xFFFFFFFF else rp.RPHYS_TERRAIN_BODY_ID)
        assert (e.position.x, e.position.y, e.position.z) == (r.point.x, r.point.y, r.point.z)
        assert e.impulse == r.impulse
