"""Shared test setup: import paths, the ``gpu`` marker, CPU checkers."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "bcm-problems_b200")
for p in (PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    from oracle_ffi import Oracle, ORACLE_SO
    if not os.path.exists(ORACLE_SO):
        pytest.fail(f"{ORACLE_SO} missing: run __graft_entry__.build()")
    return Oracle()


@pytest.fixture(scope="session")
def reflib():
    from oracle_ffi import RefLib, REF_SO
    if not os.path.exists(REF_SO):
        pytest.skip("reference library oracle/_ref not built here (needs the reference sources)")
    return RefLib()


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    import bsg
    c = bsg.Context(0)
    yield c
    c.close()
