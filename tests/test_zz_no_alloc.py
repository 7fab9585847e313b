"""rphys_ext_world_step_hash_noalloc: the tick hash with its scratch in a fixed device array.

It must return the digest rphys_world_get_step_hash returns, call after call, and allocate no
device memory once its first call on the device did the setup. Worlds beyond its stated limits are
refused with RPHYS_ERR_CAPACITY before any device work. The file sorts last so it also runs after
every other GPU test in the same process."""
import pytest

from conftest import rp, scenes

pytestmark = pytest.mark.gpu


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _check_two_in_a_row(w):
    for _ in range(2):
        assert w.hash_noalloc() == w.hash()


def test_noalloc_hash_matches_box_drop(gpu):
    w = gpu.world(1024, 1024)
    dt, _ = scenes.box_drop(rp, w, n_side=10)
    _check_two_in_a_row(w)                  # fresh world, no warm entries yet
    for t in range(90):
        w.step(dt)
        if t % 30 == 29:
            _check_two_in_a_row(w)
    assert w.stats()["warm_entries"] > 0    # the warm-start section of the stream was exercised


def test_noalloc_hash_matches_terrain(gpu):
    w = gpu.world(2048, 2048)
    dt, _ = scenes.terrain(rp, w, n_bodies=1500, hf_n=96, area=80.0)
    for _ in range(60):
        w.step(dt)
    _check_two_in_a_row(w)
    w.step(dt)
    _check_two_in_a_row(w)


def test_noalloc_hash_allocates_nothing(gpu):
    w = gpu.world(1024, 1024)
    dt, _ = scenes.box_drop(rp, w, n_side=10)
    for _ in range(30):
        w.step(dt)
    w.hash_noalloc()                        # device setup happens on the first call
    for _ in range(3):
        w.step(dt)
        before = _free_bytes()
        w.hash_noalloc()
        w.hash_noalloc()
        assert _free_bytes() == before


def test_noalloc_hash_refuses_oversized_world(gpu):
    big = gpu.world(4_500_000, 16)          # 3 bytes per body of capacity alone exceed 12 MiB
    with pytest.raises(rp.RPhysError) as e:
        big.hash_noalloc()
    assert e.value.code == rp.RPHYS_ERR_CAPACITY
    assert "at most" in e.value.msg
    big.close()
    w = gpu.world(64, 64)                   # the library stays usable
    dt, _ = scenes.box_drop(rp, w, n_side=3)
    w.step(dt)
    _check_two_in_a_row(w)


def test_noalloc_hash_with_new_joints_allocates_nothing(gpu):
    """Joints added since the last step (D6 and distance joints) are hashed without being uploaded:
    the call allocates nothing and still gives step_hash's digest, before and after stepping."""
    w = gpu.world(1024, 1024)
    dt, _, _ = scenes.ragdolls(rp, w, n_ragdolls=3)
    for _ in range(20):
        w.step(dt)
    w.hash_noalloc()                        # device setup
    a, b = w.add_box((0.0, 9.0, 0.0), (0.3, 0.3, 0.3)), w.add_box((0.0, 10.0, 0.0), (0.3, 0.3, 0.3))
    j = w.add_joints([(0, a, b, ((0.0, 0.5, 0.0), (0.0, 0.0, 0.0, 1.0)), ((0.0, -0.5, 0.0), (0.0, 0.0, 0.0, 1.0)), 0)])
    w.add_distance_joints([(a, b, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 1.0, 0.0, 0.0)])
    w.set_joint_limit(j, True, 1, -0.5, 0.5)
    before = _free_bytes()
    h_new = w.hash_noalloc()                # joints dirty: nothing uploaded, nothing allocated
    assert _free_bytes() == before
    assert h_new == w.hash()                # step_hash uploads them and gives the same digest
    for _ in range(5):
        w.step(dt)
        before = _free_bytes()
        h = w.hash_noalloc()
        assert _free_bytes() == before
        assert h == w.hash()
