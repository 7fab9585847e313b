"""The oracle against the reference's own golden bits: riftphys-world/tests/distance_bits_test.rs
records, for a box swinging on a distance joint from a static pivot (kind 0 rigid, kind 1 a spring;
3 s at 60 and 240 Hz), an FNV-1a fold of the box's final pose and velocity bits, produced by the
reference binary (lines 50-57). The oracle's restatement of the whole tick -- integration with its
gyroscopic midpoint, the joint velocity row, the SHAKE position pass, the velocity update from
corrections -- reproduces all four, which pins its arithmetic, glam's quaternion lane order
included, to the reference's. (The guard-controller scenes, kind 2, are outside the step path.)"""
import ctypes

import pytest

GOLDEN = {  # distance_bits_test.rs:52-55
    (0, 60.0): 0x87F81A83F9615530,
    (0, 240.0): 0xE7411745726C1915,
    (1, 60.0): 0x6F111D612DA3E10F,
    (1, 240.0): 0xED532E5E87913E18,
}


@pytest.mark.parametrize("kind,hz", sorted(GOLDEN))
def test_distance_joint_scene_matches_reference_bits(oracle, kind, hz):
    f = oracle.dll.rphys_oracle_distance_bits
    f.restype, f.argtypes = ctypes.c_uint64, [ctypes.c_uint32, ctypes.c_float]
    got = f(kind, hz)
    assert got == GOLDEN[(kind, hz)], f"kind {kind} {hz} Hz: {got:016x}, reference {GOLDEN[(kind, hz)]:016x}"
