"""Shared test setup: repository on sys.path, the ``gpu`` marker, and builds.

``-m "not gpu"`` tests need no GPU: the oracle against the reference's golden
outputs, the C ABI (exports, struct layout, host helpers, host-side error
paths).  ``-m gpu`` tests call libxgpu.so on a B200 and compare with the
oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    if not os.path.exists(oracle.LIB):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def xg():
    import xgpu_b200
    if not os.path.exists(xgpu_b200.LIB_PATH):
        xgpu_b200.build()
    xgpu_b200.lib()
    return xgpu_b200


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np
    d = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(d, "golden.json")) as fh:
        meta = json.load(fh)
    arrays = dict(np.load(os.path.join(d, "golden.npz")))
    return meta, arrays
