"""The reference's joint acceptance tests (joint_energy_test.rs, hinge_angle_test.rs) on the CPU oracle.
(The same cases run on the CUDA library in tests/test_gpu_joints.py.)"""
import pytest

import joint_cases as J


@pytest.mark.parametrize("name", [n for n in dir(J) if n.startswith("case_")])
def test_case(oracle, name):
    getattr(J, name)(oracle)


def test_shake_turned_threshold(oracle):
    """The GPU's position pass evaluates SHAKE's 'turned less than SHAKE_MAX_TURN' test
    (bodies.rs:486-490: 2 acos(min(|w|, 1)) < 0.5) as min(|w|, 1) >= 0x3f780aa6. The two forms agree on
    every f32 in [0.8, 1] under the project's acos; below 0.8, 2 acos exceeds 1.28 and both fail."""
    import ctypes
    f = oracle.dll.rphys_oracle_turned_threshold_mismatches
    f.restype, f.argtypes = ctypes.c_uint32, [ctypes.c_uint32]
    assert f(0x3F780AA6) == 0
    assert f(0x3F780AA5) > 0 and f(0x3F780AA7) > 0  # the neighbours of the threshold do not agree


def test_shake_max_turn_cos_bits(oracle):
    """The GPU's distance-joint position solve compares against SHAKE_MAX_TURN.cos() (bodies.rs:520)
    as the constant 0x3f60a940; the oracle computes it with the project's cosine."""
    import ctypes
    f = oracle.dll.rphys_oracle_shake_max_turn_cos_bits
    f.restype, f.argtypes = ctypes.c_uint32, []
    assert f() == 0x3F60A940
