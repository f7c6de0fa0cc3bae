"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on any host (the oracle against its pins, host logic, the
C-ABI library's exports); `-m gpu` runs the CUDA path against the oracle.
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def pq():
    import polariseq_b200 as pq_mod

    return pq_mod
