"""GPU parity: the CUDA step against the CPU oracle on the same seeded scenes, tick by tick.

Pair lists, culled manifolds (which points, in which slot order, with which solver level) and the
tick hash must be bit-identical; body states are compared bit for bit too (the two run the same
IEEE f32 operation sequence), with the divergence reported per tick if that ever fails."""
import numpy as np
import pytest

from conftest import rp, scenes

pytestmark = pytest.mark.gpu


def _records(w):
    out = []
    for c in w.contact_records():
        out.append((c.a_collider, c.b_collider, c.point.x, c.point.y, c.point.z, c.normal.x, c.normal.y, c.normal.z,
                    c.depth, c.impulse, c.level))
    return np.array(out, dtype=np.float64) if out else np.zeros((0, 11))


def run_pair(oracle, gpu, build, ticks, check_every=1):
    wo, wg = oracle.world(*build["cap"]), gpu.world(*build["cap"])
    dt, _ = build["fn"](rp, wo)
    build["fn"](rp, wg)
    for t in range(ticks):
        wo.step(dt)
        wg.step(dt)
        if t % check_every and t != ticks - 1:
            continue
        po, pg = wo.pairs(), wg.pairs()
        assert po.shape == pg.shape and np.array_equal(po, pg), f"tick {t}: pair lists differ"
        ro, rg = _records(wo), _records(wg)
        assert ro.shape == rg.shape, f"tick {t}: contact count {len(ro)} vs {len(rg)}"
        assert np.array_equal(ro[:, [0, 1, 10]], rg[:, [0, 1, 10]]), f"tick {t}: contact slots / levels differ"
        assert np.array_equal(ro.astype(np.float32).view(np.uint32), rg.astype(np.float32).view(np.uint32)), \
            f"tick {t}: contact geometry or impulse bits differ"
        so, sg = wo.body_states(), wg.body_states()
        if not np.array_equal(so.view(np.uint32), sg.view(np.uint32)):
            d = np.abs(so - sg).max()
            raise AssertionError(f"tick {t}: body state bits differ (max |diff| {d:.3e})")
        assert wo.hash() == wg.hash(), f"tick {t}: tick hash differs"
        sto, stg = wo.stats(), wg.stats()
        for k in ("pairs", "contacts", "islands", "levels", "max_batch", "warm_matched", "warm_entries", "sleeping",
                  "bounce_rows", "sweeps", "row_sweeps", "rows_scheduled", "islands_capped", "residual", "rows_capped",
                  "res_hist"):
            assert sto[k] == stg[k], f"tick {t}: stat {k} {sto[k]} vs {stg[k]}"
    return wo, wg


def test_box_drop_small(oracle, gpu):
    build = {"cap": (64, 64), "fn": lambda rp_, w: scenes.box_drop(rp_, w, n_side=3)}
    run_pair(oracle, gpu, build, 240)


def test_box_drop_1000(oracle, gpu):
    build = {"cap": (1024, 1024), "fn": lambda rp_, w: scenes.box_drop(rp_, w, n_side=10)}
    run_pair(oracle, gpu, build, 300, check_every=1)


def test_terrain_small(oracle, gpu):
    build = {"cap": (2048, 2048), "fn": lambda rp_, w: scenes.terrain(rp_, w, n_bodies=1500, hf_n=96, area=80.0)}
    run_pair(oracle, gpu, build, 200, check_every=5)


def _residual(fn, tol=1e-4, cap=80):
    def build(rp_, w):
        out = fn(rp_, w)
        w.set_residual_mode(tol, cap)
        return out
    return build


def test_box_drop_1000_residual_mode(oracle, gpu):
    # each solve island sweeps until its largest velocity change is <= 1e-4 m/s (or 32 sweeps)
    build = {"cap": (1024, 1024), "fn": _residual(lambda rp_, w: scenes.box_drop(rp_, w, n_side=10), cap=32)}
    run_pair(oracle, gpu, build, 150, check_every=10)


def test_terrain_small_residual_mode(oracle, gpu):
    build = {"cap": (2048, 2048), "fn": _residual(lambda rp_, w: scenes.terrain(rp_, w, n_bodies=1500, hf_n=96, area=80.0))}
    _, wg = run_pair(oracle, gpu, build, 160, check_every=8)
    s = wg.stats()
    assert s["rows_scheduled"] > 0 and s["row_sweeps"] < 80 * s["rows_scheduled"]  # islands stop on their own
