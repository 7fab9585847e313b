"""Coloured order on the CPU restatement (rphys_ext_set_solve_order): a valid colouring (the rows of
one colour never share a body they write), no more steps per sweep than the level schedule where
that matters, the same bits on every thread count, and results that stay near the serial order's."""
import ctypes

import numpy as np

from conftest import rp, scenes


def _terrain(lib, coloured, n=2000, threads=1):
    w = lib.world(n + 16, n + 16)
    dt, _ = scenes.terrain(rp, w, n_bodies=n, area=400.0 * (n / 100_000) ** 0.5)
    w.set_residual_mode(1e-4, 80)
    if coloured:
        w.set_coloured(True)
    lib.dll.rphys_oracle_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.dll.rphys_oracle_set_threads(w.h, threads)
    return w, dt


def _repeats(w):
    """(level, body) keys that more than one scheduled contact of the last tick holds."""
    seen = {}
    for c in w.contact_records():
        if c.level == 0xFFFFFFFF:
            continue
        for b in (c.a_collider, c.b_collider):   # one collider per body: collider index = body index
            if b != 0xFFFFFFFF:
                seen[(c.level, b)] = seen.get((c.level, b), 0) + 1
    return {k for k, v in seen.items() if v > 1}


def test_colours_share_no_written_body(oracle):
    """From the same state, the level schedule and the colouring see the same contacts; a body may
    appear twice in one colour only where it also appears twice in one level -- a body no contact
    row writes (asleep during the solve)."""
    s, dt = _terrain(oracle, False)
    for _ in range(149):
        s.step(dt)
    c, _ = _terrain(oracle, True)
    c.state_import(s.state_export())
    s.step(dt)
    c.step(dt)
    read_only = {b for _, b in _repeats(s)}
    assert c.stats()["levels"] > 1 and c.stats()["contacts"] == s.stats()["contacts"]
    for lvl, b in _repeats(c):
        assert b in read_only, f"colour {lvl}: body {b} is written by two rows of one colour"
    assert c.stats()["levels"] <= s.stats()["levels"] + 8


def test_coloured_is_deterministic_and_close_to_serial(oracle):
    a, dt = _terrain(oracle, True, threads=1)
    b, _ = _terrain(oracle, True, threads=8)
    s, _ = _terrain(oracle, False, threads=8)
    diverged = False
    for t in range(150):
        a.step(dt); b.step(dt); s.step(dt)
        assert a.hash() == b.hash(), f"tick {t}: coloured order differs between thread counts"
        diverged = diverged or a.hash() != s.hash()
    assert diverged                                   # the order is really another one
    pa, ps = a.body_states()[:, 0:3], s.body_states()[:, 0:3]
    assert np.linalg.norm(pa - ps) / np.linalg.norm(ps) < 1e-2


def test_set_solve_order_rejects_unknown(oracle):
    w, _ = _terrain(oracle, False, n=10)
    try:
        w.c("rphys_ext_set_solve_order", 7)
    except rp.RPhysError as e:
        assert e.code == rp.RPHYS_ERR_BAD_ARG
    else:
        raise AssertionError("order 7 accepted")


def test_tuning_is_stored_and_checked(oracle):
    w, _ = _terrain(oracle, False, n=10)
    assert w.tuning() == {"group_rows": 64, "packed_threads": 32, "island_threads": 128}
    w.set_tuning(16, 128, 256)
    assert w.tuning() == {"group_rows": 16, "packed_threads": 128, "island_threads": 256}
    try:
        w.set_tuning(32, 48, 128)
    except rp.RPhysError as e:
        assert e.code == rp.RPHYS_ERR_BAD_ARG
    else:
        raise AssertionError("packed_threads 48 accepted")


def test_tuning_accepts_the_tuner_grid_and_nothing_else(oracle):
    """Every launch shape the autotuner times is accepted by the C ABI's check (the CPU restatement
    applies the same check as the CUDA library), and shapes outside the grid are refused."""
    import itertools
    import riftphys_rust_b200.autotune as autotune
    w, _ = _terrain(oracle, False, n=10)
    for gr, pt, it in itertools.product(autotune.GRID["group_rows"], autotune.GRID["packed_threads"],
                                        autotune.GRID["island_threads"]):
        w.set_tuning(gr, pt, it)
        assert w.tuning() == {"group_rows": gr, "packed_threads": pt, "island_threads": it}
    for bad in [(12, 32, 32), (256, 32, 32), (0, 32, 32), (64, 256, 32), (64, 32, 512), (64, 32, 16)]:
        try:
            w.set_tuning(*bad)
        except rp.RPhysError as e:
            assert e.code == rp.RPHYS_ERR_BAD_ARG
        else:
            raise AssertionError(f"shape {bad} accepted")
    assert w.tuning() == {"group_rows": 128, "packed_threads": 128, "island_threads": 256}  # the last accepted one
