import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def svb():
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def orc():
    return __graft_entry__.load_oracle()


@pytest.fixture(scope="session")
def net(svb):
    return svb.weights.load_model()


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def golden_meta():
    with open(os.path.join(GOLDEN, "golden_meta.json")) as f:
        return json.load(f)


def bits(a):
    """FP64 values as their bit patterns, for bit-exact comparisons."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64)).view(np.uint64)
