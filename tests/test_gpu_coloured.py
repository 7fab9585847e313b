"""Coloured order on the GPU (rphys_ext_set_solve_order(RPHYS_ORDER_COLOURED)).

* Bit parity with the CPU restatement in coloured order: the 1,000-box drop, the terrain scene in
  residual mode, and a batch whose pyramid is solved by the big-island kernel.
* The divergence from the reference's serial order on the terrain generator (full 512^2
  heightfield, 12,500 bodies at the workload's density) over the configured 600 ticks: per tick, one
  coloured tick from the serial run's state against the serial tick (relative L2 difference of
  positions, linear and angular velocities), and the free-running coloured trajectory against the
  serial one. The report prints with -s."""
import numpy as np
import pytest

from conftest import rp, scenes
from test_gpu_parity import run_pair

pytestmark = pytest.mark.gpu


def _coloured(fn):
    def build(rp_, w):
        out = fn(rp_, w)
        w.set_coloured(True)
        return out
    return build


def test_coloured_box_drop_matches_oracle(oracle, gpu):
    build = {"cap": (1024, 1024), "fn": _coloured(lambda rp_, w: scenes.box_drop(rp_, w, n_side=10))}
    run_pair(oracle, gpu, build, 200, check_every=5)


def test_coloured_terrain_residual_matches_oracle(oracle, gpu):
    def fn(rp_, w):
        out = scenes.terrain(rp_, w, n_bodies=1500, hf_n=96, area=80.0)
        w.set_residual_mode(1e-4, 80)
        return out
    build = {"cap": (2048, 2048), "fn": _coloured(fn)}
    run_pair(oracle, gpu, build, 160, check_every=4)


def test_coloured_batch_big_island_matches_oracle(oracle, gpu):
    descs = [scenes.batch_world_descs(rp, 0, n_min=700, n_max=800)]
    descs += [scenes.batch_world_descs(rp, k, n_min=16, n_max=200) for k in range(1, 6)]
    total = sum(len(d) for d in descs)
    b = gpu.world(total + 8, total + 8)
    dt = scenes.batch_setup(b)
    b.set_coloured(True)
    for d in descs:
        b.add_world(d)
    ows = []
    for d in descs:
        o = oracle.world(len(d), len(d))
        scenes.batch_setup(o)
        o.set_coloured(True)
        o.add_bodies_array(d)
        ows.append(o)
    for t in range(60):
        b.step(dt)
        for o in ows:
            o.step(dt)
        hs = b.world_hashes()
        for k, o in enumerate(ows):
            assert hs[k] == o.hash(), f"tick {t}: world {k} hash differs"


def _rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


def test_coloured_divergence_from_serial_order_over_600_ticks(gpu):
    n = 12_500
    area = 400.0 * (n / 100_000) ** 0.5

    def world(coloured):
        w = gpu.world(n + 16, n + 16)
        dt, _ = scenes.terrain(rp, w, n_bodies=n, area=area)
        if coloured:
            w.set_coloured(True)
        return w, dt
    ser, dt = world(False)
    col, _ = world(True)     # free-running coloured trajectory
    one, _ = world(True)     # one coloured tick from the serial state
    per_tick, levels = [], []
    for t in range(600):
        one.state_import(ser.state_export())
        ser.step(dt)
        one.step(dt)
        col.step(dt)
        s1, s0 = one.body_states(), ser.body_states()
        per_tick.append((_rel(s1[:, 0:3], s0[:, 0:3]), _rel(s1[:, 7:10], s0[:, 7:10]), _rel(s1[:, 10:13], s0[:, 10:13])))
        levels.append((ser.stats()["levels"], one.stats()["levels"]))
    per_tick = np.array(per_tick)
    traj = _rel(col.body_states()[:, 0:3], ser.body_states()[:, 0:3])
    lv = np.array(levels)
    print(f"\n[coloured] per-tick relative divergence from the serial order (pos, lin, ang): "
          f"median {np.median(per_tick, axis=0)}, max {per_tick.max(axis=0)}; positions after 600 free-running "
          f"ticks {traj:.3e}; levels (serial, coloured) mean {lv.mean(axis=0)}, max {lv.max(axis=0)}")
    assert lv[:, 1].max() <= lv[:, 0].max()
    assert np.median(per_tick[:, 0]) < 1e-4
