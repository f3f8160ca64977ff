"""The oracle's three-body + self velocities against golden vectors from the reference's own
model classes (python/HIGNN/model_structure.py:41-139; tests/golden/make_three_body_golden.py).
CPU only."""
import os

import numpy as np
import pytest

from oracle import hignn_oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "three_body_velocity.npz")


@pytest.fixture(scope="module")
def nets():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from hignn_b200.weights import default_three_body_paths

    p3, ps = default_three_body_paths()
    return O.DenseTanh.from_hgnw(p3), O.DenseTanh.from_hgnw(ps)


@pytest.mark.parametrize("case", ["filaments", "dense"])
def test_three_body_velocity_matches_reference(case, nets):
    g = np.load(GOLD)
    u = O.three_body_velocity(g[f"{case}_x"], g[f"{case}_f"], float(g[f"{case}_eps"]), *nets)
    ref64, ref32 = g[f"{case}_v64"], g[f"{case}_v32"]
    # the FP64 golden differences positions in FP64, the oracle (like the FP32 reference) in float32
    assert np.linalg.norm(u - ref64) / np.linalg.norm(ref64) < 1e-7
    assert np.linalg.norm(u - ref32) / np.linalg.norm(ref64) < 2e-6  # the reference's FP32 path
