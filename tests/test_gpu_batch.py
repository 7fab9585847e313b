"""Batched worlds: many independent worlds stepped together in one RPhysWorld on the GPU, each
checked against its own CPU-restatement World built from the same bodies (capacity = its body
count). Per-world tick hashes, body states and pair lists must be bit-identical, and a restore of
the batch snapshot must replay every world's hashes."""
import numpy as np
import pytest

from conftest import rp, scenes

pytestmark = pytest.mark.gpu


def _build(oracle, gpu, n_worlds, n_min, n_max, residual=None):
    descs = [scenes.batch_world_descs(rp, k, n_min=n_min, n_max=n_max) for k in range(n_worlds)]
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
    if residual:
        b.set_residual_mode(*residual)
        for o in ows:
            o.set_residual_mode(*residual)
    return b, ows, descs, dt


def _check(b, ows, descs, t):
    hs = b.world_hashes()
    states = b.body_states()
    pairs = b.pairs()
    c0 = 0
    for k, (o, d) in enumerate(zip(ows, descs)):
        assert hs[k] == o.hash(), f"tick {t}: world {k} hash differs"
        so = o.body_states()
        sg = states[c0:c0 + len(d)]
        assert np.array_equal(so.view(np.uint32), sg.view(np.uint32)), f"tick {t}: world {k} body states differ"
        po = o.pairs()
        mine = pairs[(pairs[:, 0] >= c0) & (pairs[:, 0] < c0 + len(d))] - c0 if len(pairs) else pairs
        assert np.array_equal(po, mine), f"tick {t}: world {k} pairs differ"
        c0 += len(d)


def test_batch_worlds_match_separate_worlds(oracle, gpu):
    b, ows, descs, dt = _build(oracle, gpu, 8, 16, 160)
    assert b.num_worlds() == 8
    for t in range(120):
        b.step(dt)
        for o in ows:
            o.step(dt)
        if t % 10 == 9:
            _check(b, ows, descs, t)


def test_batch_residual_mode_matches(oracle, gpu):
    b, ows, descs, dt = _build(oracle, gpu, 6, 16, 120, residual=(1e-4, 64))
    for t in range(90):
        b.step(dt)
        for o in ows:
            o.step(dt)
        if t % 15 == 14:
            _check(b, ows, descs, t)


def test_batch_rollback_replays_every_world(gpu):
    # rphys_ext_snapshot_restore_exact puts back every stored bit; the v1 restore re-injects poses
    # through set_pose (renormalised rotations), as the reference FFI does
    descs = [scenes.batch_world_descs(rp, k, n_min=16, n_max=200) for k in range(10)]
    total = sum(len(d) for d in descs)
    b = gpu.world(total + 8, total + 8)
    dt = scenes.batch_setup(b)
    for d in descs:
        b.add_world(d)
    for _ in range(30):
        b.step(dt)
    snap = b.snapshot()
    first = []
    for _ in range(8):
        b.step(dt)
        first.append(b.world_hashes())
    b.restore_exact(snap)
    for k in range(8):
        b.step(dt)
        assert b.world_hashes() == first[k], f"replayed tick {k} differs"
    b.free_snapshot(snap)
