"""Test configuration: the `gpu` marker, import paths, and the oracle build.

`-m "not gpu"` runs on a CPU-only machine (the oracle, the host logic, the
C-ABI symbol table); `-m gpu` needs a B200 and calls the CUDA library
through its C-ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "aeolus.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libaeolus_b200.so")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    from oracle import oracle
    if not os.path.exists(oracle.LIB_PATH):
        oracle.build()
    yield
