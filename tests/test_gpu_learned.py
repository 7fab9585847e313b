"""The learned warm start in the tick: bit-exact against the CPU restatement when the restatement
is offered the same predictions, training data export, and what a trained model gains."""
import numpy as np
import pytest

from conftest import rp, scenes

pytestmark = pytest.mark.gpu


def _terrain(lib, n=1500):
    w = lib.world(n + 16, n + 16)
    dt, _ = scenes.terrain(rp, w, n_bodies=n, hf_n=96, area=80.0)
    return w, dt


def test_learned_ticks_match_the_restatement(oracle, gpu):
    wg, dt = _terrain(gpu)
    wo, _ = _terrain(oracle)
    for _ in range(60):
        wg.step(dt)
        wo.step(dt)
    m = gpu.model(seed=11)                 # untrained: many rows fall back, some keep the prediction
    wg.set_warm_model(m)
    used = 0
    for t in range(40):
        wg.step(dt)
        p = wg.row_predictions()
        assert len(p) == wg.stats()["contacts"]
        wo.oracle_set_predictions(p)
        wo.step(dt)
        sg, so = wg.stats(), wo.stats()
        assert sg["pred_used"] == so["pred_used"], t
        used += sg["pred_used"]
        a, b = wg.body_states(), wo.body_states()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"tick {t}: body states differ"
        assert wg.hash() == wo.hash(), f"tick {t}: hash differs"
    assert used > 0


def test_feature_rows_are_logged(gpu):
    w, dt = _terrain(gpu, 800)
    w.set_feature_logging(True)
    for _ in range(80):
        w.step(dt)
    f, t = w.row_features()
    assert len(f) > 100 and f.shape[1] == 24 and t.shape[1] == 3
    assert np.isfinite(f).all() and np.isfinite(t).all()
    n = f[:, 0:3]
    assert np.allclose((n * n).sum(1), 1.0, atol=1e-4)    # unit normals
    assert (t[:, 0] >= 0).all()                          # normal impulses are non-negative


def test_trained_model_against_previous_tick_warm_start(gpu):
    # the recipe: rows logged from the plain solver, targets clipped to +-20 impulse units, trained on
    # the rows with no previous impulse (new contacts), offered to those rows only; measured as the
    # velocity row updates the residual stop needs over the same 40 ticks, with and without it
    w, dt = _terrain(gpu, 1500)
    w.set_residual_mode(1e-4, 80)
    w.set_feature_logging(True)
    feats, targs = [], []
    for t in range(220):
        w.step(dt)
        if t >= 40:
            f, tt = w.row_features()
            feats.append(f); targs.append(tt)
    F, T = np.concatenate(feats), np.concatenate(targs)
    cold = F[:, 22] == 0
    F, T = F[cold], np.clip(T[cold], -20.0, 20.0)
    m = gpu.model(seed=2)
    _, l0 = m.gradients(F[:4096], T[:4096])
    m.train(F, T, epochs=6, batch=2048, lr=1e-3)
    _, l1 = m.gradients(F[:4096], T[:4096])
    assert l1 < 0.8 * l0, (l0, l1)
    snap = w.snapshot()
    sweeps = {}
    for mode in ("previous-tick", "learned"):
        w.restore_exact(snap)
        w.set_warm_model(m if mode == "learned" else None)
        w.set_warm_policy(True)
        tot = used = conv = 0
        for _ in range(40):
            w.step(dt)
            st = w.stats()
            tot += st["row_sweeps"]
            used += st["pred_used"]
            conv += st["row_sweeps"] - 80 * st["rows_capped"]  # updates of the islands that converged
        sweeps[mode] = (tot, used, conv)
    w.set_warm_model(None)
    w.free_snapshot(snap)
    gain = 1.0 - sweeps["learned"][0] / sweeps["previous-tick"][0]
    gain_conv = 1.0 - sweeps["learned"][2] / max(1, sweeps["previous-tick"][2])
    print(f"row updates over 40 ticks (total, from prediction, in converged islands): {sweeps}; gain {100 * gain:.2f}% "
          f"overall, {100 * gain_conv:.2f}% in the islands that converge")
    assert sweeps["learned"][1] > 0
    # What the trained network gains, measured: nothing that matters. About +0.5% fewer row updates
    # on this scene; on the 100k-body bench state +0.2% with this policy. The sweeps go to islands
    # whose contact sets are infeasible and run to the cap whatever their start. In the islands that
    # converge, the previous tick's impulse is already a close start. The per-row fallback keeps a
    # prediction only where it starts the row better, so the check is that it costs no more than 2%.
    assert gain > -0.02, sweeps
