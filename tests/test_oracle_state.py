"""The state blob (rphys_ext_state_export / _import) on the CPU restatement: a world that imports
another world's blob mid-run continues bit for bit like the world it came from, and blobs of
another world are refused with nothing changed."""
import pytest

from conftest import rp, scenes


def _terrain(lib, n=600):
    w = lib.world(n + 16, n + 16)
    dt, _ = scenes.terrain(rp, w, n_bodies=n, hf_n=64, area=40.0)
    w.set_residual_mode(1e-4, 40)
    return w, dt


def test_state_blob_continues_bit_for_bit(oracle):
    a, dt = _terrain(oracle)
    for _ in range(60):
        a.step(dt)
    blob = a.state_export()
    b, _ = _terrain(oracle)
    assert b.hash() != a.hash()
    b.state_import(blob)
    assert b.hash() == a.hash()
    assert b.tick() == a.tick()
    assert b.state_export() == blob
    for t in range(20):
        a.step(dt)
        b.step(dt)
        assert a.hash() == b.hash(), f"tick {t}: hash differs after the import"


def test_state_blob_with_joints(oracle):
    def build():
        w = oracle.world(256, 256)
        dt, _, _ = scenes.ragdolls(rp, w, n_ragdolls=4)
        return w, dt
    a, dt = build()
    for _ in range(40):
        a.step(dt)
    b, _ = build()
    b.state_import(a.state_export())
    for t in range(15):
        a.step(dt)
        b.step(dt)
        assert a.hash() == b.hash(), f"tick {t}: hash differs after the import"


def test_state_blob_refuses_another_world(oracle):
    a, dt = _terrain(oracle, 600)
    a.step(dt)
    other, _ = _terrain(oracle, 500)
    h = other.hash()
    with pytest.raises(rp.RPhysError) as e:
        other.state_import(a.state_export())
    assert e.value.code == rp.RPHYS_ERR_BAD_ARG
    with pytest.raises(rp.RPhysError) as e:
        a.state_import(a.state_export()[:-1])
    assert e.value.code == rp.RPHYS_ERR_BAD_ARG
    assert other.hash() == h
