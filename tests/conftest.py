import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

WEIGHTS = os.path.join(REPO, "hignn_b200", "data", "two_body_unbounded.hgnw")
GOLDEN = os.path.join(REPO, "tests", "golden", "two_body_net.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session")
def oracle_net():
    from oracle import hignn_oracle as O

    return O.TwoBody.from_hgnw(WEIGHTS)


@pytest.fixture(scope="session")
def oracle_net_exact():
    """The oracle network whose FP32 evaluation reproduces the plain device network bit for bit."""
    from oracle import hignn_oracle as O

    return O.TwoBodyF32Exact.from_hgnw(WEIGHTS)


@pytest.fixture(scope="session")
def small_workload():
    from hignn_b200 import synthetic as S

    x = S.uniform_min_dist(4096, 0.05, 0)
    f = S.sedimenting_forces(4096, 0)
    return x, f
