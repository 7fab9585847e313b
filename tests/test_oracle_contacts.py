"""rphys_world_get_contacts on the CPU restatement: the cases of tests/contact_cases.py."""
import pytest

import contact_cases as CC


@pytest.mark.parametrize("name", [n for n in dir(CC) if n.startswith("case_")])
def test_case(oracle, name):
    getattr(CC, name)(oracle)
