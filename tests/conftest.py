"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def oracle():
    from pyoracle import Oracle, build_oracle
    build_oracle()
    return Oracle()


@pytest.fixture(scope="session")
def reflib():
    from pyoracle import RefLib, ref_available
    if not ref_available():
        pytest.skip("oracle/_ref (the reference's own CPU build) is not present")
    return RefLib()


@pytest.fixture(scope="session")
def lib():
    import stipple_b200
    from stipple_b200 import build
    build.build()
    return stipple_b200.load()


@pytest.fixture(scope="session")
def ctx(lib):
    import stipple_b200 as sb
    if sb.device_count() < 1:
        pytest.fail("no CUDA device: GPU tests need a B200")
    c = sb.Context(0)
    yield c
    c.close()
