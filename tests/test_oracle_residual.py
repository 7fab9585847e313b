"""Why some solve islands of the terrain workload never reach the 1e-4 residual.

On the terrain scene at the workload's body density (5,000 bodies in a 179 m square of the 512^2
heightfield), 200 ticks in, the CPU restatement keeps the island with the largest last-sweep
residual (an oracle-only diagnostic). Its worst rows are the terrain contacts of one body whose
capsule or sphere end sank below the surface: the reference's sphere-triangle narrowphase takes
each contact normal from the closest point on a triangle to the sunken centre
(crates/riftphys-collision/src/narrowphase.rs:671-707), so the triangles around it give normals
that point against each other, one of them down. No velocity separates the body from all of them,
the contact LCP has no solution, and projected Gauss-Seidel adds the same impulse to those rows in
every sweep: the residual stays near its first-sweep value for all 80 sweeps while the normal
impulses grow to hundreds of times the body's weight impulse. This is the reference's formulation,
restated; the GPU library gives the same bits."""
import ctypes
import os

import numpy as np

from conftest import rp, scenes


def test_worst_island_is_an_infeasible_terrain_contact_set(oracle):
    d = oracle.dll
    d.rphys_oracle_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
    d.rphys_oracle_diag_worst.argtypes = [ctypes.c_void_p, ctypes.c_int]
    d.rphys_oracle_diag_read.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                         ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                                         ctypes.POINTER(ctypes.c_uint32)]
    n = 5000
    w = oracle.world(n + 16, n + 16)
    dt, _ = scenes.terrain(rp, w, n_bodies=n, area=400.0 * (n / 100_000) ** 0.5)
    w.set_residual_mode(1e-4, 80)
    d.rphys_oracle_set_threads(w.h, os.cpu_count() or 1)
    w.step_n(dt, 199)
    d.rphys_oracle_diag_worst(w.h, 1)
    w.step_n(dt, 1)
    s = w.stats()
    assert s["islands_capped"] > 0 and s["sweeps"] == 80
    nr, nh = ctypes.c_uint32(0), ctypes.c_uint32(0)
    d.rphys_oracle_diag_read(w.h, None, 0, None, 0, ctypes.byref(nr), ctypes.byref(nh))
    rows = np.zeros((nr.value, 5), np.float32)
    hist = np.zeros(nh.value, np.float32)
    d.rphys_oracle_diag_read(w.h, rows.ctypes.data, nr.value, hist.ctypes.data, nh.value, ctypes.byref(nr),
                             ctypes.byref(nh))
    assert len(hist) == 80 and hist[-1] == s["residual"]
    # the residual barely moves over the sweeps: the same velocity change every sweep
    assert hist[-1] > 0.5 * hist[1] and hist[-1] > 0.1
    ab = rows[:, :2].view(np.uint32)
    worst = int(np.argmax(rows[:, 4]))
    body = int(ab[worst, 0])
    assert ab[worst, 1] == 0xFFFFFFFF                     # a terrain contact
    # that body's terrain contacts: opposing normals, impulses far beyond its weight impulse
    normals = np.array([(c.normal.x, c.normal.y, c.normal.z) for c in w.contact_records()
                        if c.a_collider == body and c.b_collider == 0xFFFFFFFF])
    assert len(normals) >= 2
    assert (normals @ normals.T).min() < -0.5
    assert normals[:, 1].min() < 0.0                      # one of them points down, into the ground
    m_n, jn = rows[worst, 2], rows[worst, 3]
    assert jn > 100.0 * m_n * 9.81 / 60.0
