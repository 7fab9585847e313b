"""The reference's FFI contract, determinism, rollback and acceptance tests, on the CPU oracle.
(The same cases run on the CUDA library in tests/test_gpu_abi.py.)"""
import pytest

import abi_cases as C


@pytest.fixture(scope="module")
def lib(oracle):
    return oracle


@pytest.mark.parametrize("name", [n for n in dir(C) if n.startswith("case_") and n != "case_rollback_replays"])
def test_case(lib, name):
    getattr(C, name)(lib)


@pytest.mark.parametrize("settle,asleep", [(15, False), (400, True)])
def test_rollback_replays(lib, settle, asleep):
    C.case_rollback_replays(lib, settle, asleep)
