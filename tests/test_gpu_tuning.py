"""Launch shapes of the velocity solve (rphys_ext_set_tuning) change no result bit: the terrain scene
in residual mode and a batch with a big pyramid step to the same tick hashes under shapes at both
ends of the tuner's grid; unsupported shapes are refused."""
import pytest

from conftest import rp, scenes

pytestmark = pytest.mark.gpu

SHAPES = [(64, 32, 128), (32, 32, 64), (8, 32, 32), (16, 128, 256), (32, 64, 128), (64, 32, 32), (64, 128, 64), (128, 32, 128)]


def _terrain_hashes(gpu, shape):
    w = gpu.world(3016, 3016)
    dt, _ = scenes.terrain(rp, w, n_bodies=3000, hf_n=128, area=110.0)
    w.set_residual_mode(1e-4, 80)
    w.set_tuning(*shape)
    assert tuple(w.tuning().values()) == shape
    out = []
    for _ in range(150):
        w.step(dt)
        out.append(w.hash())
    w.close()
    return out


def test_launch_shapes_keep_the_bits(gpu):
    ref = _terrain_hashes(gpu, SHAPES[0])
    for shape in SHAPES[1:]:
        assert _terrain_hashes(gpu, shape) == ref, shape


def test_unsupported_shape_is_refused(gpu):
    w = gpu.world(8, 8)
    with pytest.raises(rp.RPhysError) as e:
        w.set_tuning(12, 64, 128)
    assert e.value.code == rp.RPHYS_ERR_BAD_ARG
    assert w.tuning() == {"group_rows": 64, "packed_threads": 32, "island_threads": 128}  # the tuned defaults
