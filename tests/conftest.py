"""Shared test setup.

Tests marked `gpu` call the CUDA library through its C-ABI and compare with
the CPU oracle (oracle/) and the golden fixtures (tests/golden/, produced
from the reference itself by tests/golden/make_golden.py).  Everything else
runs on the CPU.
"""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (os.path.join(ROOT, "cu-xmss_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")
    config.addinivalue_line("markers", "slow: CPU test that takes more than ~30 s")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def xb():
    import xmss_b200

    return xmss_b200


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    if name.endswith(".json"):
        with open(path) as f:
            return json.load(f)
    with open(path) as f:
        return [l.strip() for l in f if l.strip()]


@pytest.fixture(scope="session")
def golden():
    return load_golden
