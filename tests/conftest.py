"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and the built
sm_100a library; every other test runs on the CPU."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built sm_100a library")


@pytest.fixture(scope="session")
def oracle():
    from oracle.binding import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.binding import Reference, reference_available
    if not reference_available():
        pytest.skip("reference not compiled here (oracle/_ref needs the reference sources)")
    return Reference()


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "reference_outputs.npz")))


@pytest.fixture(scope="session")
def known():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def gpu_lib():
    """The loaded library on a machine with a GPU (fails, never skips)."""
    from sparkit_b200 import gpu
    assert gpu.device_count() > 0, "no CUDA device visible"
    return gpu
