"""GPU parity at the configured sizes.

* The terrain workload at full size (100,000 bodies on the 512^2 heightfield, residual mode as
  benchmarked): the GPU steps it 240 ticks into the contact-rich regime, its state blob
  (rphys_ext_state_export) is loaded into a CPU-restatement world built from the same scene, and
  both then step on; pair lists, contact records, body states, statistics and the tick hash must be
  bit-identical every tick.
* The terrain generator on its full 512^2 heightfield at the workload's body density (12,500 bodies
  in a 141 m square), stepped in lockstep for the configured 600 ticks at 20 iterations: the hash
  every tick, everything every 30 ticks.
* A batch of worlds whose pyramid is one island of more than 1,152 rows, the class solved by the
  big-island kernel, against per-world CPU worlds."""
import ctypes
import os

import numpy as np
import pytest

from conftest import rp, scenes
from test_gpu_parity import _records

pytestmark = pytest.mark.gpu


def _threads(oracle, w):
    oracle.dll.rphys_oracle_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
    oracle.dll.rphys_oracle_set_threads(w.h, os.cpu_count() or 1)


def _compare(wo, wg, t):
    po, pg = wo.pairs(), wg.pairs()
    assert po.shape == pg.shape and np.array_equal(po, pg), f"tick {t}: pair lists differ"
    ro, rg = _records(wo), _records(wg)
    assert ro.shape == rg.shape, f"tick {t}: contact count {len(ro)} vs {len(rg)}"
    assert np.array_equal(ro.astype(np.float32).view(np.uint32), rg.astype(np.float32).view(np.uint32)), \
        f"tick {t}: contact records differ"
    so, sg = wo.body_states(), wg.body_states()
    if not np.array_equal(so.view(np.uint32), sg.view(np.uint32)):
        raise AssertionError(f"tick {t}: body state bits differ (max |diff| {np.abs(so - sg).max():.3e})")
    assert wo.hash() == wg.hash(), f"tick {t}: tick hash differs"
    sto, stg = wo.stats(), wg.stats()
    for k in ("pairs", "contacts", "islands", "levels", "max_batch", "warm_matched", "warm_entries", "sleeping",
              "sweeps", "row_sweeps", "rows_scheduled", "islands_capped", "residual", "rows_capped", "res_hist"):
        assert sto[k] == stg[k], f"tick {t}: stat {k} {sto[k]} vs {stg[k]}"


def test_terrain_100k_on_512_from_the_gpu_state(oracle, gpu):
    n = 100_000
    wg, wo = gpu.world(n + 16, n + 16), oracle.world(n + 16, n + 16)
    dt, _ = scenes.terrain(rp, wg, n_bodies=n)
    scenes.terrain(rp, wo, n_bodies=n)
    for w in (wg, wo):
        w.set_residual_mode(1e-4, 80)
    _threads(oracle, wo)
    wg.step_n(dt, 240)
    wo.state_import(wg.state_export())
    assert wo.hash() == wg.hash(), "tick 240: hash of the imported state differs"
    for t in range(241, 244):
        wg.step(dt)
        wo.step(dt)
        _compare(wo, wg, t)
    s = wg.stats()
    assert s["contacts"] > 300_000 and s["islands"] > 10_000   # the contact-rich regime the bench times


def test_terrain_512_for_600_ticks(oracle, gpu):
    n = 12_500
    area = 400.0 * (n / 100_000) ** 0.5
    wg, wo = gpu.world(n + 16, n + 16), oracle.world(n + 16, n + 16)
    dt, _ = scenes.terrain(rp, wg, n_bodies=n, area=area)
    scenes.terrain(rp, wo, n_bodies=n, area=area)
    _threads(oracle, wo)
    for t in range(600):
        wg.step(dt)
        wo.step(dt)
        if t % 30 == 29 or t == 599:
            _compare(wo, wg, t)
        else:
            assert wo.hash() == wg.hash(), f"tick {t}: tick hash differs"
    assert wg.stats()["contacts"] > 20_000


def test_batch_big_island_matches_separate_worlds(oracle, gpu):
    descs = [scenes.batch_world_descs(rp, 0, n_min=700, n_max=800)]           # a pyramid, one island
    descs += [scenes.batch_world_descs(rp, k, n_min=16, n_max=200) for k in range(1, 6)]
    total = sum(len(d) for d in descs)
    b = gpu.world(total + 8, total + 8)
    dt = scenes.batch_setup(b)
    for d in descs:
        b.add_world(d)
    ows = []
    for d in descs:
        o = oracle.world(len(d), len(d))
        scenes.batch_setup(o)
        o.add_bodies_array(d)
        ows.append(o)
    big = 0
    for t in range(60):
        b.step(dt)
        for o in ows:
            o.step(dt)
        big = max(big, b.stats()["max_group_rows"])
        hs = b.world_hashes()
        for k, o in enumerate(ows):
            assert hs[k] == o.hash(), f"tick {t}: world {k} hash differs"
        if t % 10 == 9:
            states, c0 = b.body_states(), 0
            for k, (o, d) in enumerate(zip(ows, descs)):
                sg = states[c0:c0 + len(d)]
                assert np.array_equal(o.body_states().view(np.uint32), sg.view(np.uint32)), \
                    f"tick {t}: world {k} body states differ"
                c0 += len(d)
    assert big > 1152, f"the pyramid never reached the big-island class (largest group {big} rows)"

