"""The reference's joint acceptance tests (joint_energy_test.rs, hinge_angle_test.rs) on the CPU oracle.
(The same cases run on the CUDA library in tests/test_gpu_joints.py.)"""
import pytest

import joint_cases as J


@pytest.mark.parametrize("name", [n for n in dir(J) if n.startswith("case_")])
def test_case(oracle, name):
    getattr(J, name)(oracle)
